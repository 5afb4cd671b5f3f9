// Newton-Schulz inverse of an N x N complex matrix on tcgen05 tensor cores (TF32 operands, FP32
// accumulators in TMEM), one CTA:
//     X_{k+1} = X_k (2 I - B X_k),   I - B X_{k+1} = (I - B X_k)^2,
// which converges quadratically from any seed X_0 with spectral radius rho(I - B X_0) < 1.  Every
// complex product is two real MMA groups with M = 128 (rows >= N are padding), N_pad = N rounded
// up to 16 columns, K = 2 N:
//     Re(P Q) = Pr Qr - Pi Qi  ->  A = Pr then Pi, B = Qr^T then -Qi^T (the B-negate bit)
//     Im(P Q) = Pr Qi + Pi Qr  ->  A = Pr then Pi, B = Qi^T then Qr^T
// written to TMEM columns [0, N_pad) and [64, 64 + N_pad).  Thread t < N owns row t: after each
// product it reads its row from TMEM in chunks of 16 columns, forms the next operand (Z = 2 I - Y,
// or the new X) and writes it back to shared memory in the layouts the next product reads (rows of
// X for A, columns of X or Z for B).  Nothing crosses threads except through the tensor core and
// one block-wide maximum per iteration.
//
// Stopping: after Y = B X_k the CTA takes e_k = max_i sum_j (|Re| + |Im|)(I - Y)_ij.  If e_k^2 <= tol
// (or the iteration limit is reached) X_{k+1} is the result; e_k >= 1 (or not finite) means the
// seed was too far: the iteration stops and reports failure, and the caller inverts another way.
//
// Shared memory (NsSmem<N>::bytes, 128-byte aligned): six N x N FP32 operand buffers
// [Br | Bi | Xr | Xi | Tr | Ti] in the K-major layout of tc05.cuh (R = N rows), then 128 bytes the
// B reads of the last buffer may touch.  The M = 128 reads of every A buffer run up to 1408 bytes
// past its end, into the buffers that follow it.
#pragma once

#include "tc05.cuh"

namespace ns {

template <int N>
struct NsSmem {
    static_assert(N % 16 == 8 || N % 16 == 0, "row groups of 8");
    static_assert(N <= 64, "TMEM columns [0, 64) and [64, 128) per part");
    static constexpr int NP = (N + 15) / 16 * 16;                 // MMA N (a multiple of 16)
    static constexpr uint32_t buf = (uint32_t)N * N * 4;          // one operand buffer
    static constexpr uint32_t off_br = 0, off_bi = buf, off_xr = 2 * buf, off_xi = 3 * buf, off_tr = 4 * buf,
                              off_ti = 5 * buf;
    static constexpr uint32_t bytes = (6 * buf + 128 + 127) / 128 * 128;
    static constexpr uint32_t lbo = (uint32_t)(N / 8) * 128;       // next column group (4 elements of K)
    static constexpr uint32_t sbo = 128;                           // next row group (8 rows)
    static constexpr uint32_t tmem_cols = 128;
};

constexpr int kNsMaxPolls = 1 << 22;   // bounded mbarrier wait (well under a second)

// One complex product into TMEM: D_re = A_r Q_r - A_i Q_i at column 0, D_im = A_r Q_i + A_i Q_r at
// column 64.  a_r, a_i: A buffers (rows of the left factor); q_r, q_i: B buffers (columns of the
// right factor).  Issued by one thread; the caller commits.
template <int N>
__device__ __forceinline__ void issue_cplx(uint32_t tmem, uint32_t a_r, uint32_t a_i, uint32_t q_r, uint32_t q_i) {
    using S = NsSmem<N>;
    constexpr uint32_t id_pos = tc05::idesc_tf32(128, S::NP, false);
    constexpr uint32_t id_neg = tc05::idesc_tf32(128, S::NP, true);
#pragma unroll
    for (int s = 0; s < N / 8; ++s) {   // K = 8 per instruction: column groups 2 s, 2 s + 1
        const uint32_t ko = (uint32_t)(2 * s) * S::lbo;
        const uint64_t ar = tc05::smem_desc(a_r + ko, S::lbo, S::sbo), ai = tc05::smem_desc(a_i + ko, S::lbo, S::sbo);
        const uint64_t br = tc05::smem_desc(q_r + ko, S::lbo, S::sbo), bi = tc05::smem_desc(q_i + ko, S::lbo, S::sbo);
        tc05::mma_tf32(tmem, ar, br, id_pos, s > 0);          // + A_r Q_r
        tc05::mma_tf32(tmem, ai, bi, id_neg, true);           // - A_i Q_i
        tc05::mma_tf32(tmem + 64, ar, bi, id_pos, s > 0);     // + A_r Q_i
        tc05::mma_tf32(tmem + 64, ai, br, id_pos, true);      // + A_i Q_r
    }
}

// 16 columns [c, c + 16) of this thread's TMEM lane, real part (column c) and imaginary part
// (column 64 + c); whole warp
__device__ __forceinline__ void load_chunk(uint32_t taddr_lane, int c, float (&re)[16], float (&im)[16]) {
    tc05::tmem_ld16(taddr_lane + c, re);
    tc05::tmem_ld16(taddr_lane + 64 + c, im);
    tc05::tmem_wait_ld();
}

// element (t, k) of an A buffer (row t) and element (n, t) of a B buffer (column t), TF32-rounded
template <int N>
__device__ __forceinline__ void store_a4(unsigned char* buf, int t, int k, float v0, float v1, float v2, float v3) {
    *reinterpret_cast<float4*>(buf + tc05::kmajor_offset(N, t, k)) =
        make_float4(tc05::to_tf32f(v0), tc05::to_tf32f(v1), tc05::to_tf32f(v2), tc05::to_tf32f(v3));
}
template <int N>
__device__ __forceinline__ void store_b(unsigned char* buf, int t, int n, float v) {
    *reinterpret_cast<float*>(buf + tc05::kmajor_offset(N, n, t)) = tc05::to_tf32f(v);
}

struct NsState {
    uint32_t tmem;       // TMEM base (lane 0, column base)
    uint32_t phase;      // parity of the next mbarrier phase
    bool ok;             // every wait completed
};

// Wait for the product committed last, then make TMEM readable.  On a wait that runs out the state
// is marked failed; nothing more is issued and the caller frees TMEM after a bounded drain.
__device__ __forceinline__ void wait_product(NsState& st, uint64_t* bar) {
    const bool done = tc05::mbar_wait(bar, st.phase, kNsMaxPolls);
    st.phase ^= 1u;
    st.ok = st.ok && done;
    tc05::fence_after();
}

// Before the caller frees TMEM: if a wait ran out, give the product in flight one more bounded wait.
__device__ __forceinline__ void drain(NsState& st, uint64_t* bar) {
    if (!st.ok) (void)tc05::mbar_wait(bar, st.phase, kNsMaxPolls);
}

// Issue one complex product after the operands' shared-memory writes (all threads call this).
template <int N>
__device__ __forceinline__ void product(NsState& st, uint64_t* bar, uint32_t a_r, uint32_t a_i, uint32_t q_r,
                                        uint32_t q_i) {
    tc05::fence_async_smem();
    tc05::fence_before();
    __syncthreads();
    if (threadIdx.x == 0 && st.ok) {
        tc05::fence_after();
        issue_cplx<N>(st.tmem, a_r, a_i, q_r, q_i);
        tc05::commit(bar);
    }
    if (st.ok) wait_product(st, bar);
}

// Newton-Schulz iterations on buffers already holding B (Br, Bi as A operands) and the seed X_0 (Xr,
// Xi as A operands; Tr, Ti its columns as B operands), written and not yet fenced.  All threads of
// the CTA call it.  emit(t, c, re, im) receives the result's row t, columns [c, c + 16) (entries >= N
// unspecified) for every t < N.  red: >= blockDim.x / 32 floats of scratch.  Returns true when the
// result met e^2 <= tol with every wait completed; *err_out = the last e_k.
template <int N, class Emit>
__device__ bool newton_schulz(unsigned char* sm, uint64_t* bar, float* red, NsState& st, int max_its, float tol,
                              Emit&& emit, float* err_out) {
    using S = NsSmem<N>;
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t base = tc05::smem_addr(sm);
    const uint32_t lane_addr = st.tmem + ((uint32_t)(32 * (warp & 3)) << 16);
    constexpr int kWarps = (N + 31) / 32;     // warps whose lanes hold rows < N
    bool done = false, conv = false;
    float e_last = INFINITY;
    for (int it = 0; it < max_its && !done; ++it) {
        // ---- Y = B X_k; Z = 2 I - Y into (Tr, Ti) as B operand columns; e_k
        product<N>(st, bar, base + S::off_br, base + S::off_bi, base + S::off_tr, base + S::off_ti);
        float e = 0.f;
        if (warp < kWarps) {
#pragma unroll 1
            for (int c = 0; c < N; c += 16) {
                float yr[16], yi[16];
                load_chunk(lane_addr, c, yr, yi);
                if (tid < N) {
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        const int n = c + j;
                        if (n < N) {
                            const float dr = (n == tid ? 1.f : 0.f) - yr[j];
                            e += fabsf(dr) + fabsf(yi[j]);
                            store_b<N>(sm + S::off_tr, tid, n, dr + (n == tid ? 1.f : 0.f));
                            store_b<N>(sm + S::off_ti, tid, n, -yi[j]);
                        }
                    }
                }
            }
        }
        if (tid >= N || !(e == e)) e = tid < N ? INFINITY : 0.f;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) e = fmaxf(e, __shfl_xor_sync(0xffffffffu, e, o));
        if ((tid & 31) == 0) red[warp] = e;
        tc05::fence_before();
        __syncthreads();
        float ek = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) ek = fmaxf(ek, red[w]);
        e_last = ek;
        if (!(ek < 1.f) || !st.ok) break;                 // diverging (or a wait ran out): no result
        const bool last = ek * ek <= tol || it == max_its - 1;
        // ---- X_{k+1} = X_k Z
        product<N>(st, bar, base + S::off_xr, base + S::off_xi, base + S::off_tr, base + S::off_ti);
        if (warp < kWarps) {
#pragma unroll 1
            for (int c = 0; c < N; c += 16) {
                float xr[16], xi[16];
                load_chunk(lane_addr, c, xr, xi);
                if (tid < N) {
                    if (last) {
                        emit(tid, c, xr, xi);
                    } else {
#pragma unroll
                        for (int j = 0; j < 16; j += 4)
                            if (c + j < N) {
                                store_a4<N>(sm + S::off_xr, tid, c + j, xr[j], xr[j + 1], xr[j + 2], xr[j + 3]);
                                store_a4<N>(sm + S::off_xi, tid, c + j, xi[j], xi[j + 1], xi[j + 2], xi[j + 3]);
                            }
#pragma unroll
                        for (int j = 0; j < 16; ++j)
                            if (c + j < N) {
                                store_b<N>(sm + S::off_tr, tid, c + j, xr[j]);
                                store_b<N>(sm + S::off_ti, tid, c + j, xi[j]);
                            }
                    }
                }
            }
        }
        if (last) {
            done = true;
            conv = st.ok && ek * ek <= tol;
        }
    }
    tc05::fence_before();
    // every TMEM read of this CTA is complete; red may be reused; the verdict is the CTA's
    const bool all = __syncthreads_and(conv ? 1 : 0) != 0;
    if (err_out) *err_out = e_last;
    return all;
}

}  // namespace ns
