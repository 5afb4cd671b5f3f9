// tcgen05 (fifth-generation tensor core) building blocks for sm_100a: tensor-memory (TMEM)
// allocation, the shared-memory and instruction descriptors of tcgen05.mma, the MMA issue, its
// completion through an mbarrier, and TMEM loads.
//
// Operand layout used here (no swizzle, K-major): a matrix of R rows (R a multiple of 8) and K
// columns of 32-bit elements is stored as "core matrices" of 8 rows x 4 elements (16 bytes per
// row, 128 contiguous bytes).  Core matrix (row group rg, column group kg) starts at
//     rg * 128 + kg * (R / 8) * 128
// bytes: the row groups of one column group are adjacent (the descriptor's stride byte offset,
// SBO = 128) and column groups follow each other (leading byte offset, LBO = R / 8 * 128).  One
// kind::tf32 instruction consumes K = 8 (two column groups); its descriptor starts at column group
// 2 s.  An M = 128 instruction reads 16 row groups per column group: where only the first R < 128
// rows carry data, the other row groups alias the next column groups (or up to 15 * 128 bytes
// past the buffer's end), whose values only reach output rows >= R, which are never read.
//
// Accumulator layout (cta_group::1, M = 128, 32-bit): row m of D is TMEM lane m, column n is TMEM
// column (base + n).  Warp w of a warpgroup reads lanes 32 (w % 4) .. 32 (w % 4) + 31.
//
// Field positions follow the PTX ISA's descriptor tables (shared-memory descriptor: start address,
// LBO, SBO in 16-byte units at bits 0, 16, 32, version 1 at bit 46, layout type at bits 61..63;
// instruction descriptor: D format at bit 4, A / B formats at bits 7 / 10, negate bits 13 / 14,
// N / 8 at bit 17, M / 16 at bit 24).
#pragma once

#include <cstdint>

namespace tc05 {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// byte offset of element (r, k) in the K-major no-swizzle layout above (R rows)
__host__ __device__ constexpr uint32_t kmajor_offset(int R, int r, int k) {
    return (uint32_t)((r >> 3) * 128 + (k >> 2) * (R / 8) * 128 + (r & 7) * 16 + (k & 3) * 4);
}

// shared-memory matrix descriptor: K-major, no swizzle
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;   // descriptor version of sm_100
    return d;                 // base offset 0, absolute LBO mode, layout type 0 (no swizzle)
}

// instruction descriptor of kind::tf32: D in FP32, A and B TF32, both K-major; neg_b negates B
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N, bool neg_b = false) {
    return (1u << 4) | (2u << 7) | (2u << 10) | (neg_b ? (1u << 14) : 0u) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A B^T for one K = 8 slice; issued by one thread
__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         bool accumulate) {
    const uint32_t acc = accumulate ? 1u : 0u, z = 0u;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}

// the mbarrier at bar receives one arrival once every MMA issued before by this thread completed
__device__ __forceinline__ void commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :
                 : "r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes become visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" : : "r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// bounded wait for the phase with the given parity; false when the limit ran out
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int max_polls) {
    const uint32_t a = smem_addr(bar);
    for (int i = 0; i < max_polls; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// TMEM allocation of ncols columns (a power of two >= 32) by one whole warp; the base address is
// written to *slot (shared memory)
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :
                 : "r"(smem_addr(slot)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t base, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" : : "r"(base), "r"(ncols) : "memory");
}

// 16 consecutive 32-bit columns of this thread's TMEM lane (whole warp; lane base in bits 16..31)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ float to_tf32f(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

}  // namespace tc05
