// a5/a6 (F, lambda_0), a8/a11-a13 (Matsubara sums, lambda_m Newton) and a15 (mu fit, G_ladder,
// energies).
//
// The reductions and root finders run on one 8-CTA thread-block cluster: every Newton iteration's
// sums are reduced inside each CTA, exchanged through distributed shared memory after a hardware
// cluster barrier, and added in rank order by every CTA, which then takes the same Newton step.
// No host round trip sits between iterations, the inputs (lambda, rhs, lambda_min) can come from
// device memory written earlier on the stream, and the summation order is fixed, so reruns are
// bitwise identical.
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include "ldga_internal.cuh"

namespace cg = cooperative_groups;

namespace {

constexpr int kCluster = 8;
constexpr int kClThreads = 512;

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Shared state of cluster_sum: per-warp partials, two exchange slots read by the other CTAs of the
// cluster (alternating between calls), and the broadcast of the totals inside the CTA.
template <int NV>
struct ClRed {
    double red[NV * 32];
    double part[2 * NV];
    double bcast[NV];
};

// Cluster-wide sums of NV values in a fixed order; every thread of every CTA receives the totals.
// Per call: warp shuffles, one CTA barrier, warp 0 folds the warp partials and publishes them, one
// cluster barrier, then warp 0 alone reads the kCluster remote partials (one distributed-shared-
// memory load per lane) and broadcasts the totals through shared memory.  Slot reuse is safe: a
// slot written in call i + 2 was last read before every CTA arrived at the barrier of call i + 1.
// parity: a register of every thread, flipped identically by all of them.
template <int NV>
__device__ void cluster_sum(double (&v)[NV], ClRed<NV>& s, int& parity) {
    cg::cluster_group cl = cg::this_cluster();
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nwarp = blockDim.x >> 5;
    const int slot = parity * NV;
#pragma unroll
    for (int j = 0; j < NV; ++j) v[j] = warp_sum(v[j]);
    if (l == 0) {
#pragma unroll
        for (int j = 0; j < NV; ++j) s.red[j * 32 + w] = v[j];
    }
    __syncthreads();
    if (w == 0) {
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            const double x = warp_sum(l < nwarp ? s.red[j * 32 + l] : 0.0);
            if (l == 0) s.part[slot + j] = x;
        }
    }
    cl.sync();
    if (w == 0) {
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            const double x = warp_sum(l < kCluster ? cl.map_shared_rank(s.part, l)[slot + j] : 0.0);
            if (l == 0) s.bcast[j] = x;
        }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < NV; ++j) v[j] = s.bcast[j];
    parity ^= 1;
}

// One-barrier cluster all-reduce for loops that reduce every iteration (Newton).  Each warp folds
// its NV values with shuffles and lanes 0..kCluster-1 store them into slot [parity] of every CTA of
// the cluster (lane r writes CTA r); after one cluster barrier every warp of every CTA sums all
// kCluster * warps partials itself, in the same fixed order, so all threads hold identical totals
// with no further CTA barrier.  A slot written in call i + 2 was last read before every thread
// arrived at the barrier of call i + 1.
constexpr int kClWarps = kClThreads / 32;
// The lambda_m Newton runs 256 threads per CTA: its cost per iteration is the all-reduce, and
// fewer warps mean fewer partials to exchange and add (measured 0.162 vs 0.172 ms for 100
// iterations on 39 729 points, 8 x 256 vs 8 x 512 threads).
constexpr int kNewtonThreads = 256;
template <int NV, int NW = kClWarps, int CL = kCluster>
struct ClAll {
    // [slot][source warp][value]: a source's NV values are adjacent, so NV = 2 moves as one
    // 16-byte remote store and one 16-byte shared load
    alignas(16) double part[2][CL * NW][NV];
};

template <int NV, int NW, int CL>
__device__ __forceinline__ void cluster_allsum(double (&v)[NV], ClAll<NV, NW, CL>& s, int& parity) {
    cg::cluster_group cl = cg::this_cluster();
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    const int src = (int)cl.block_rank() * NW + w;
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        double x = v[j];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        v[j] = x;
    }
    if (l < CL) {
        ClAll<NV, NW, CL>* dst = cl.map_shared_rank(&s, l);
        if constexpr (NV == 2) {
            *reinterpret_cast<double2*>(dst->part[parity][src]) = make_double2(v[0], v[1]);
        } else {
#pragma unroll
            for (int j = 0; j < NV; ++j) dst->part[parity][src][j] = v[j];
        }
    }
    cl.sync();
    constexpr int P = CL * NW;
    double x[NV];
#pragma unroll
    for (int j = 0; j < NV; ++j) x[j] = 0.0;
#pragma unroll
    for (int i = l; i < P; i += 32) {
        if constexpr (NV == 2) {
            const double2 p = *reinterpret_cast<const double2*>(s.part[parity][i]);
            x[0] += p.x;
            x[1] += p.y;
        } else {
#pragma unroll
            for (int j = 0; j < NV; ++j) x[j] += s.part[parity][i][j];
        }
    }
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        for (int o = 16; o > 0; o >>= 1) x[j] += __shfl_xor_sync(0xffffffffu, x[j], o);
        v[j] = x[j];
    }
    parity ^= 1;
}

// The same all-reduce without a cluster barrier.  Lanes 0..kCluster-1 of every warp write the warp's
// NV values into CTA l's slot with st.async, which completes its bytes on that CTA's mbarrier of the
// slot; each CTA arms its own mbarrier for the bytes of all kCluster * NW sources (one arrive with
// expect_tx by thread 0) and its threads wait for that phase -- no release fence over the cluster and
// no barrier that every CTA must reach.  Slot s of a CTA is rewritten (iteration i + 2) only after
// every source received this CTA's iteration i + 1 values, which each warp sends after it has read
// slot s (its shuffles of iteration i); the mbarrier of slot s advances one phase per use, so the
// waiters of iteration i see phase parity (i / 2) & 1.  Waits are bounded: after kAsyncSpins
// non-blocking polls (mbarrier.test_wait, well under a second) the call returns false and the caller
// stops its loop and reports NaN.
constexpr long long kAsyncSpins = 1ll << 22;

template <int NV, int NW, int CL = kCluster>
struct ClAsync {
    alignas(16) double part[2][CL * NW][NV];
    alignas(8) unsigned long long bar[2];
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

template <int NV, int NW, int CL>
__device__ __forceinline__ void async_allsum_init(ClAsync<NV, NW, CL>& s) {
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&s.bar[0])), "r"(1) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&s.bar[1])), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    cg::this_cluster().sync();   // every CTA's barriers exist before any remote write
}

template <int NV, int NW, int CL>
__device__ __forceinline__ bool async_allsum(double (&v)[NV], ClAsync<NV, NW, CL>& s, int iter) {
    static_assert(NV == 2, "the exchange moves one 16-byte value pair per source");
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    const int slot = iter & 1;
    const uint32_t phase = (uint32_t)((iter >> 1) & 1);
    const uint32_t src = cg::this_cluster().block_rank() * NW + w;
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        double x = v[j];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        v[j] = x;
    }
    const uint32_t bar = smem_addr(&s.bar[slot]);
    if (threadIdx.x == 0) {
        constexpr uint32_t bytes = CL * NW * NV * sizeof(double);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
    }
    if (l < CL) {
        uint32_t raddr, rbar;
        asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(raddr) : "r"(smem_addr(&s.part[slot][src][0])), "r"(l));
        asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(rbar) : "r"(bar), "r"(l));
        asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.f64 [%0], {%1, %2}, [%3];"
                     ::"r"(raddr), "d"(v[0]), "d"(v[1]), "r"(rbar) : "memory");
    }
    uint32_t done = 0;
    for (long long k = 0; k < kAsyncSpins && !done; ++k)
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}" : "=r"(done) : "r"(bar), "r"(phase) : "memory");
    const bool ok = __all_sync(0xffffffffu, done != 0);
    constexpr int P = CL * NW;
    double x[NV];
#pragma unroll
    for (int j = 0; j < NV; ++j) x[j] = 0.0;
#pragma unroll
    for (int i = l; i < P; i += 32) {
        const double2 p = *reinterpret_cast<const double2*>(s.part[slot][i]);
        x[0] += p.x;
        x[1] += p.y;
    }
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        for (int o = 16; o > 0; o >>= 1) x[j] += __shfl_xor_sync(0xffffffffu, x[j], o);
        v[j] = x[j];
    }
    return ok;
}

__device__ __forceinline__ int cl_tid() { return cg::this_cluster().block_rank() * blockDim.x + threadIdx.x; }
__device__ __forceinline__ int cl_nth() { return kCluster * blockDim.x; }

// ---------------------------------------------------------------------------------------------
// F_from_χ (BSETools.jl:40-53) and lambda_0 (BSETools.jl:129-141)
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ double2 gimp_at(const double2* g, int n) { return n >= 0 ? g[n] : cconj(g[-n - 1]); }

__global__ void k_F_from_chi(int nnu, int nw, int n_iv, int n_iw, int shift, double beta,
                             const double2* __restrict__ chi, const double2* __restrict__ gimp,
                             double2* __restrict__ F) {
    const int total = nnu * nnu * nw;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        const int vi = e % nnu, r = e / nnu, vpi = r % nnu, wi = r / nnu;
        const int wn = wi - n_iw;
        const int vn = (vi - n_iv) - shift * (wn / 2);
        const int vpn = (vpi - n_iv) - shift * (wn / 2);
        const double2 g1 = gimp_at(gimp, vn), g2 = gimp_at(gimp, wn + vn);
        const double2 g3 = gimp_at(gimp, vpn), g4 = gimp_at(gimp, wn + vpn);
        double2 num = chi[e];
        if (vn == vpn) num = cadd(num, cscale(cmul(g1, g2), beta));
        const double2 den = cmul(cmul(cmul(g1, g2), g3), g4);
        const double2 v = cdiv(num, den);
        F[e] = make_double2(-v.x, -v.y);
    }
}

// colF[nu', w] = sum_nu F[nu, nu', w]: one warp per column (nu', w), coalesced loads, then a fixed-order
// shuffle reduction (bitwise reproducible).  A thread per column summed its 40 values one dependent
// load after another.
__global__ void k_colsum_F(int nnu, int nw, const double2* __restrict__ F, double2* __restrict__ colF) {
    const int lane = threadIdx.x & 31;
    const int ncol = nnu * nw, nwarp_all = (gridDim.x * blockDim.x) >> 5;
    for (int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < ncol; c += nwarp_all) {
        const double2* col = F + (size_t)c * nnu;
        double2 acc = make_double2(0.0, 0.0);
        for (int v = lane; v < nnu; v += 32) acc = cadd(acc, col[v]);
        for (int o = 16; o > 0; o >>= 1) {
            acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
            acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
        }
        if (lane == 0) colF[c] = acc;
    }
}

__global__ void k_lambda0(int nq, int nnu, int nw, double inv_beta2, const double2* __restrict__ chi0,
                          const double2* __restrict__ colF, double2* __restrict__ l0) {
    const size_t total = (size_t)nq * nnu * nw;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const size_t vw = e / nq;
        l0[e] = cscale(cmul(chi0[e], colF[vw]), inv_beta2);
    }
}

// adjoint of k_lambda0 with respect to chi0: chi0_bar += lambda0_bar conj(colF) / beta^2
__global__ void k_lambda0_vjp(int nq, int nnu, int nw, double inv_beta2, const double2* __restrict__ colF,
                              const double2* __restrict__ l0_bar, double2* __restrict__ chi0_bar) {
    const size_t total = (size_t)nq * nnu * nw;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const size_t vw = e / nq;
        chi0_bar[e] = cadd(chi0_bar[e], cscale(cmul(l0_bar[e], cconj(colF[vw])), inv_beta2));
    }
}

// ---------------------------------------------------------------------------------------------
// sum_kω (DataTypes.jl:230-249):  (sum_w [ sum_q kMult f(chi)/N_k - c2/(i w)^2 ] - beta^2 c2/12)/beta
// ---------------------------------------------------------------------------------------------
struct SumArgs {
    int nq, nw, n_iw;
    double beta, c2, inv_nk;
};

// sum over w != 0 of real(c2/(i w_m)^2) = -c2 beta^2/(4 pi^2 m^2)
__device__ __forceinline__ double w2_tail(const SumArgs& a) {
    double tail = 0.0;
    for (int m = 1; m <= a.n_iw; ++m) tail += 2.0 * (-a.c2 * a.beta * a.beta / (4.0 * M_PI * M_PI * (double)m * m));
    return tail;
}
__device__ __forceinline__ double finish_kw(const SumArgs& a, double s) {
    return (s * a.inv_nk - w2_tail(a) + (-a.beta * a.beta / 12.0) * a.c2) / a.beta;
}

// mode 0: chi_lambda, 1: dchi_lambda, 2: sum_ωk order (per q over w first, then kMult)
__global__ void __cluster_dims__(kCluster, 1, 1) __launch_bounds__(kClThreads)
k_sum_kw(SumArgs a, const double* __restrict__ chi, const double* __restrict__ kmult, double lam,
         const double* lam_dev, int mode, double* out) {
    __shared__ ClRed<1> cr;
    int parity = 0;
    if (lam_dev) lam += lam_dev[0];
    double v[1] = {0.0};
    if (mode == 2) {
        const double tail = w2_tail(a);
        for (int q = cl_tid(); q < a.nq; q += cl_nth()) {
            double s = 0.0;
            for (int w = 0; w < a.nw; ++w) {
                const double x = chi[(size_t)w * a.nq + q];
                s += lam != 0.0 ? x / (lam * x + 1.0) : x;
            }
            s = (s - tail + a.c2 * (-a.beta * a.beta / 12.0)) / a.beta;
            v[0] = fma(kmult[q], s, v[0]);
        }
        cluster_sum<1>(v, cr, parity);
        if (cl_tid() == 0) out[0] = v[0] * a.inv_nk;
    } else {
        const int total = a.nq * a.nw;
        for (int e = cl_tid(); e < total; e += cl_nth()) {
            const int q = e % a.nq;
            const double x = chi[e];
            const double t = lam != 0.0 ? x / (lam * x + 1.0) : x;
            v[0] = fma(kmult[q], mode == 1 ? -t * t : t, v[0]);
        }
        cluster_sum<1>(v, cr, parity);
        if (cl_tid() == 0) out[0] = finish_kw(a, v[0]);
    }
    cg::this_cluster().sync();
}

__global__ void __launch_bounds__(1024) k_lambda_min(int nq, int w0, const double* chi, double* out) {
    __shared__ double red[33];
    double mn = INFINITY;
    for (int q = threadIdx.x; q < nq; q += blockDim.x) mn = fmin(mn, 1.0 / chi[(size_t)w0 * nq + q]);
    for (int o = 16; o > 0; o >>= 1) mn = fmin(mn, __shfl_down_sync(0xffffffffu, mn, o));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) red[w] = mn;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = INFINITY;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) r = fmin(r, red[i]);
        out[0] = -r;
    }
}

// newton_right, 1-D (LambdaCorrection/helpers.jl:133-153), iteration for iteration; f and df are the
// reference's f_c1/df_c1 (conditions_new.jl:152-153): both carry the tail terms of sum_kω.
// rhs = rhs_const - (rhs_sub ? rhs_sub[0] : 0); xmin = get_λ_min(chi), formed at the start (below).
// K > 0: every thread keeps its K elements of chi and their kMult weights in registers for the whole
// loop (elements e = tid + j * threads, the order the K = 0 streaming form sums in); the constant
// tail of sum_kω is formed once.  An iteration is then one or two divisions (the batch inversion
// below), one cluster_allsum and the step.
//
// Periodic trajectories are shortened exactly.  Near the root |f| often stays above atol (1e-13 is
// below the rounding noise of the sum), so newton_right runs all nsteps iterations while xi hops
// among a few values ulps apart.  The state (x0, xi) at the top of an iteration fixes every later
// iteration (the sums are reduced in a fixed order, so f and df are bitwise reproducible), so once
// that state equals the one saved at the last power-of-two checkpoint (iterations 1, 2, 4, ...),
// the trajectory has period p = i - checkpoint and whole periods up to nsteps are skipped; the last
// < p iterations then run as usual.  xi and i come out bit for bit as from the full loop.
// out[3], out[4]: the iteration at which the repeat was recognised and p (0, 0: nothing skipped).
//
// CL: CTAs of the cluster, given at launch (cudaLaunchAttributeClusterDimension).  16 (a non-portable
// size, where the GPU can place it) halves each thread's share of the sums against 8; the exchange
// costs the same number of steps either way, one st.async per lane and a wider final fold.
//
// xmin = get_λ_min(chi) = -min_q 1/chi(q, ω0) (LambdaCorrection/helpers.jl:217-220) is formed by every
// CTA from the nq values of column w0 (a CTA-local min: fmin is exact, so every CTA gets the same
// value bit for bit, the value k_lambda_min gives), and CTA 0 stores it to xmin_out.
template <int K, bool ASYNC, int CL>
__global__ void __launch_bounds__(kNewtonThreads)
k_lambda_m(SumArgs a, const double* __restrict__ chi, const double* __restrict__ kmult, double rhs_const,
           const double* rhs_sub, int w0, double* xmin_out, int nsteps, double atol, double* out,
           const double* __restrict__ chi_d, double* sum_d_out, double* sum_m_out) {
    __shared__ ClAll<2, kNewtonThreads / 32, CL> ca;
    __shared__ ClAsync<2, kNewtonThreads / 32, CL> cs;
    __shared__ double s_min[kNewtonThreads / 32];
    int parity = 0, iter = 0;
    bool exchange_ok = true;
    {
        double mn = INFINITY;
        for (int q = threadIdx.x; q < a.nq; q += blockDim.x) mn = fmin(mn, 1.0 / chi[(size_t)w0 * a.nq + q]);
        for (int o = 16; o > 0; o >>= 1) mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        if ((threadIdx.x & 31) == 0) s_min[threadIdx.x >> 5] = mn;
    }
    if constexpr (ASYNC) async_allsum_init(cs);   // its cluster barrier also orders s_min
    else __syncthreads();
    double xmin;
    {
        double mn = INFINITY;
        for (int i = 0; i < kNewtonThreads / 32; ++i) mn = fmin(mn, s_min[i]);
        xmin = -mn;
    }
    if (cg::this_cluster().block_rank() == 0 && threadIdx.x == 0) xmin_out[0] = xmin;
    auto allsum = [&](double (&v)[2]) -> bool {
        if constexpr (ASYNC) return async_allsum(v, cs, iter++);
        cluster_allsum<2>(v, ca, parity);
        return true;
    };
    const double delta = 1e-4;
    const int total = a.nq * a.nw;
    const int tid = cl_tid(), nth = CL * (int)blockDim.x;
    // finish_kw(s) = (s inv_nk - tail + c) / beta with the tail and constant hoisted out of the loop
    const double tail = w2_tail(a);
    const double cst = (-a.beta * a.beta / 12.0) * a.c2;
    const double inv_beta = 1.0 / a.beta;             // the step's /beta as one product
    double xv[K > 0 ? K : 1], kv[K > 0 ? K : 1];
#pragma unroll
    for (int j = 0; j < K; ++j) {
        const int e = tid + j * nth;
        xv[j] = e < total ? chi[e] : 0.0;
        kv[j] = e < total ? kmult[e % a.nq] : 0.0;
    }
    // the chain's rhs = rhs_const - sum_kω(chi_d) formed here (chi_d given) instead of by a k_sum_kw
    // launch before the Newton; the same elements and weights as the chi_m sums below
    double rhs = rhs_const - (rhs_sub ? rhs_sub[0] : 0.0);
    if (chi_d) {
        double v[2] = {0.0, 0.0};
        for (int e = tid; e < total; e += nth) v[0] = fma(kmult[e % a.nq], chi_d[e], v[0]);
        if (!allsum(v)) exchange_ok = false;
        const double sd = (v[0] * a.inv_nk - tail + cst) * inv_beta;
        rhs = rhs_const - sd;
        if (tid == 0 && sum_d_out) sum_d_out[0] = sd;
    }
    double x0 = 0.0, xi = x0;
    int i = 1;
    long long ck_x0 = __double_as_longlong(x0), ck_xi = __double_as_longlong(xi);
    int ck_i = 1, skip_at = 0, skip_p = 0;
    while (true) {
        double v[2] = {0.0, 0.0};
        if (K > 0) {
            // Batch inversion (Montgomery's trick): prefix products of the denominators 1 + xi x,
            // one division of the total, then every 1/d_j from two products.  The direct form's
            // K divisions ran one after another, each behind its slow-path branch; these products
            // overlap.  K > 8 splits into two independent batches (two divisions, shorter chains,
            // fewer live registers).  A product outside [1e-300, 1e300] (an exact pole, extreme
            // lambda) takes the direct divisions, so infinities stay confined to their elements.
            constexpr int NB = K > 8 ? 2 : 1;
            constexpr int G = (K + NB - 1) / NB;
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                constexpr int G0 = G > 0 ? G : 1;
                double d[G0], pre[G0];
                double prod = 1.0;
#pragma unroll
                for (int u = 0; u < G; ++u) {
                    const int j = b * G + u;
                    d[u] = j < K ? fma(xi, xv[j < K ? j : 0], 1.0) : 1.0;
                    pre[u] = prod;
                    prod *= d[u];
                }
                double s0 = 0.0, s1 = 0.0;       // per-batch partial sums: independent chains
                if (fabs(prod) > 1e-300 && fabs(prod) < 1e300) {
                    double r = 1.0 / prod;
#pragma unroll
                    for (int u = G - 1; u >= 0; --u) {
                        const int j = b * G + u;
                        const double inv = r * pre[u];
                        r *= d[u];
                        if (j < K) {
                            const double t = xv[j] * inv;
                            s0 = fma(kv[j], t, s0);
                            s1 = fma(kv[j], -t * t, s1);
                        }
                    }
                } else {
#pragma unroll
                    for (int u = 0; u < G; ++u) {
                        const int j = b * G + u;
                        if (j < K) {
                            const double t = xv[j] / d[u];
                            s0 = fma(kv[j], t, s0);
                            s1 = fma(kv[j], -t * t, s1);
                        }
                    }
                }
                v[0] += s0;
                v[1] += s1;
            }
        } else {
            for (int e = tid; e < total; e += nth) {
                const double x = chi[e];
                const double t = x / (xi * x + 1.0);
                const double km = kmult[e % a.nq];
                v[0] = fma(km, t, v[0]);
                v[1] = fma(km, -t * t, v[1]);
            }
        }
        if (!exchange_ok || !allsum(v)) { exchange_ok = false; xi = NAN; break; }
        const double fi = (v[0] * a.inv_nk - tail + cst) * inv_beta - rhs;
        const double dfi = (v[1] * a.inv_nk - tail + cst) * inv_beta;
        const double dfii = 1.0 / dfi;
        xi = x0 - dfii * fi;
        if (fabs(fi) < atol) break;
        if (xi < xmin) x0 = xmin + delta + fabs(xmin - x0) / 2.0;
        else x0 = xi;
        if (i >= nsteps) break;
        ++i;
        // top of iteration i: every thread holds the same (x0, xi), so the branch is uniform
        const long long bx0 = __double_as_longlong(x0), bxi = __double_as_longlong(xi);
        if (skip_p == 0 && bx0 == ck_x0 && bxi == ck_xi) {
            skip_at = i;
            skip_p = i - ck_i;
            i += skip_p * ((nsteps - i) / skip_p);
        } else if (skip_p == 0 && (i & (i - 1)) == 0) {
            ck_x0 = bx0;
            ck_xi = bxi;
            ck_i = i;
        }
    }
    // the chain's sum_kω(chi_m) at the final λ (the EoM's tail term), instead of a k_sum_kw launch after
    if (sum_m_out) {
        double v[2] = {0.0, 0.0};
        for (int e = tid; e < total; e += nth) {
            const double x = chi[e];
            v[0] = fma(kmult[e % a.nq], xi != 0.0 ? x / (xi * x + 1.0) : x, v[0]);
        }
        if (exchange_ok && !allsum(v)) exchange_ok = false;
        if (tid == 0) sum_m_out[0] = exchange_ok ? (v[0] * a.inv_nk - tail + cst) * inv_beta : NAN;
    }
    if (tid == 0) {
        out[0] = exchange_ok ? xi : NAN;   // an exchange that timed out leaves no valid λ
        out[1] = (double)i;
        out[3] = (double)skip_at;
        out[4] = (double)skip_p;
    }
    cg::this_cluster().sync();
}

// ---------------------------------------------------------------------------------------------
// mu fit (G_from_Σladder!, GFTools.jl:162-186 with filling_pos :255-273) and calc_E
// (thermodynamics.jl:142-168) for the Sigma_ladder on the device.
// ---------------------------------------------------------------------------------------------
struct GArgs {
    int nq, numax;
    double beta, U, n, inv_nk, shell;
};

__device__ __forceinline__ double2 g_at(double mu, double eps, double2 sig, int nn, double beta) {
    // 1/(i nu_n + mu - eps - Sigma)
    return cinv(make_double2(mu - eps - sig.x, (2.0 * nn + 1.0) * M_PI / beta - sig.y));
}

// K > 0: the Newton loop keeps every thread's K (q, nu) elements (kMult, eps_q, Sigma, nu_n) in
// registers; K = 0 streams them from memory each iteration.
//
// CL CTAs of NT threads, the cluster size given at launch.  CL = 16 (NT = 256, where the device can
// place the non-portable size; the λm Newton's choice) exchanges the sums by st.async into every
// CTA's shared memory with mbarrier completion (async_allsum) and halves each thread's elements;
// CL = 8 (NT = 512) keeps one cluster barrier per exchange.
template <int K, int CL, int NT>
__global__ void __launch_bounds__(NT)
k_mu_fit_energy(GArgs a, const double* __restrict__ kmult, const double* __restrict__ eps,
                const double2* __restrict__ sigma, int fix_n, double mu_in, const double* mu_dev, double* out) {
    constexpr bool ASYNC = CL != kCluster;
    __shared__ ClAll<2, NT / 32, CL> ca2;
    __shared__ ClAsync<2, NT / 32, CL> xs;
    __shared__ ClRed<3> cr3;
    int parity = 0, iter = 0;
    bool exchange_ok = true;
    if constexpr (ASYNC) async_allsum_init(xs);
    auto allsum = [&](double (&v)[2]) {
        if constexpr (ASYNC) { if (!async_allsum(v, xs, iter++)) exchange_ok = false; }
        else cluster_allsum<2>(v, ca2, parity);
    };
    const int total = a.nq * a.numax;
    const int cl_n = CL * (int)blockDim.x;
    double mu = mu_dev ? mu_dev[0] : mu_in;   // the start: a value written earlier on the stream, or mu_in
    bool failed = false;
    double ck[K > 0 ? K : 1], ce[K > 0 ? K : 1], cw[K > 0 ? K : 1];
    double2 cs[K > 0 ? K : 1];
    if (fix_n) {
#pragma unroll
        for (int j = 0; j < K; ++j) {
            const int e = cl_tid() + j * cl_n;
            const bool in = e < total;
            const int q = in ? e % a.nq : 0, nn = in ? e / a.nq : 0;
            ck[j] = in ? kmult[q] : 0.0;       // padding elements carry weight 0
            ce[j] = in ? eps[q] : 0.0;
            cs[j] = in ? sigma[e] : make_double2(0.0, 0.0);
            cw[j] = (2.0 * nn + 1.0) * M_PI / a.beta;
        }
    }
    if (fix_n) {
        // safeguarded Newton (same method as the oracle's mu_newton); f = filling_pos - n
        double lo = -INFINITY, hi = INFINITY;
        const double tol = 1e-14;
        for (int it = 0; it < 100; ++it) {
            double v[2] = {0.0, 0.0};
            if (K > 0) {
#pragma unroll
                for (int j = 0; j < K; ++j) {
                    // g_at(mu, eps, sigma, nn, beta) with its operands from registers
                    const double2 G = cinv(make_double2(mu - ce[j] - cs[j].x, cw[j] - cs[j].y));
                    v[0] = fma(ck[j], G.x, v[0]);
                    v[1] = fma(ck[j], -(G.x * G.x - G.y * G.y), v[1]);
                }
            } else {
                for (int e = cl_tid(); e < total; e += cl_n) {
                    const int q = e % a.nq, nn = e / a.nq;
                    const double2 G = g_at(mu, eps[q], sigma[e], nn, a.beta);
                    v[0] = fma(kmult[q], G.x, v[0]);
                    v[1] = fma(kmult[q], -(G.x * G.x - G.y * G.y), v[1]);
                }
            }
            allsum(v);
            if (!exchange_ok) { failed = true; break; }
            const double sG = v[0] * a.inv_nk, dG = v[1] * a.inv_nk;
            const double f = 2.0 * (2.0 * sG / a.beta + 0.5 + mu * a.shell) / (1.0 + a.U * a.shell) - a.n;
            const double df = 2.0 * (2.0 * dG / a.beta + a.shell) / (1.0 + a.U * a.shell);
            if (!isfinite(f)) { failed = true; break; }
            if (fabs(f) < tol) break;
            if (f > 0) hi = fmin(hi, mu); else lo = fmax(lo, mu);
            const double step = df != 0.0 ? f / df : 0.0;
            double nw = mu - step;
            if (!(lo < nw && nw < hi) || !isfinite(nw)) {
                if (isfinite(lo) && isfinite(hi)) nw = 0.5 * (lo + hi);
                else nw = mu - (f > 0 ? 1.0 : (f < 0 ? -1.0 : 0.0)) * fmax(1.0, fabs(step));
            }
            if (fabs(nw - mu) <= 1e-15 * (1.0 + fabs(mu))) { mu = nw; break; }
            mu = nw;
        }
    }
    if (failed) mu = NAN;
    // energies at mu (calc_E with the fitted mu) and the filling
    const double hartree = a.n * a.U / 2.0;
    double v[3] = {0.0, 0.0, 0.0};
    for (int e = cl_tid(); e < total; e += cl_n) {
        const int q = e % a.nq, nn = e / a.nq;
        const double2 G = g_at(mu, eps[q], sigma[e], nn, a.beta);
        const double wn = (2.0 * nn + 1.0) * M_PI / a.beta;
        const double tail = -1.0 / (wn * wn);                           // 1/(i w)^2
        const double ekin_tc = eps[q] + hartree - mu;
        const double epot_tc = a.U * a.U * 0.5 * a.n * (1.0 - 0.5 * a.n) + hartree * (eps[q] + hartree - mu);
        const double2 GS = cmul(G, sigma[e]);
        v[0] = fma(kmult[q], 4.0 * (eps[q] * (G.x - ekin_tc * tail)), v[0]);
        v[1] = fma(kmult[q], 2.0 * (GS.x - epot_tc * tail), v[1]);
        v[2] = fma(kmult[q], G.x, v[2]);
    }
    for (int q = cl_tid(); q < a.nq; q += cl_n) {     // tail_inv terms, once per q
        const double ekin_tc = eps[q] + hartree - mu;
        const double epot_tc = a.U * a.U * 0.5 * a.n * (1.0 - 0.5 * a.n) + hartree * (eps[q] + hartree - mu);
        v[0] = fma(kmult[q], (a.beta / 2.0) * eps[q] * (1.0 + -a.beta * ekin_tc), v[0]);
        v[1] = fma(kmult[q], (a.beta / 2.0) * hartree + (a.beta / 2.0) * (-a.beta / 2.0) * epot_tc, v[1]);
    }
    if constexpr (ASYNC) {
        double v01[2] = {v[0], v[1]}, v2[2] = {v[2], 0.0};
        allsum(v01);
        allsum(v2);
        v[0] = v01[0];
        v[1] = v01[1];
        v[2] = v2[0];
        if (!exchange_ok) v[0] = v[1] = v[2] = NAN;
    } else {
        cluster_sum<3>(v, cr3, parity);
    }
    if (cl_tid() == 0) {
        const double sG = v[2] * a.inv_nk;
        out[0] = mu;
        out[1] = v[0] * a.inv_nk / a.beta;
        out[2] = v[1] * a.inv_nk / a.beta;
        out[3] = 2.0 * (2.0 * sG / a.beta + 0.5 + mu * a.shell) / (1.0 + a.U * a.shell);
    }
    cg::this_cluster().sync();
}

// calc_E for a given G (column stride ldg) and Sigma over nu_n = 0..numax-1 (thermodynamics.jl:142-168)
__global__ void __cluster_dims__(kCluster, 1, 1) __launch_bounds__(kClThreads)
k_calc_E(GArgs a, const double* kmult, const double* eps, const double2* G, int ldg, const double2* sigma,
         double mu, double* out) {
    __shared__ ClRed<2> cr;
    int parity = 0;
    const double hartree = a.n * a.U / 2.0;
    double v[2] = {0.0, 0.0};
    const int total = a.nq * a.numax;
    for (int e = cl_tid(); e < total; e += cl_nth()) {
        const int q = e % a.nq, nn = e / a.nq;
        const double2 g = G[(size_t)nn * ldg + q];
        const double wn = (2.0 * nn + 1.0) * M_PI / a.beta;
        const double tail = -1.0 / (wn * wn);
        const double ekin_tc = eps[q] + hartree - mu;
        const double epot_tc = a.U * a.U * 0.5 * a.n * (1.0 - 0.5 * a.n) + hartree * (eps[q] + hartree - mu);
        const double2 GS = cmul(g, sigma[e]);
        v[0] = fma(kmult[q], 4.0 * (eps[q] * (g.x - ekin_tc * tail)), v[0]);
        v[1] = fma(kmult[q], 2.0 * (GS.x - epot_tc * tail), v[1]);
    }
    for (int q = cl_tid(); q < a.nq; q += cl_nth()) {
        const double ekin_tc = eps[q] + hartree - mu;
        const double epot_tc = a.U * a.U * 0.5 * a.n * (1.0 - 0.5 * a.n) + hartree * (eps[q] + hartree - mu);
        v[0] = fma(kmult[q], (a.beta / 2.0) * eps[q] * (1.0 + -a.beta * ekin_tc), v[0]);
        v[1] = fma(kmult[q], (a.beta / 2.0) * hartree + (a.beta / 2.0) * (-a.beta / 2.0) * epot_tc, v[1]);
    }
    cluster_sum<2>(v, cr, parity);
    if (cl_tid() == 0) { out[0] = v[0] * a.inv_nk / a.beta; out[1] = v[1] * a.inv_nk / a.beta; }
    cg::this_cluster().sync();
}

// G_ladder over fft_range: Sigma_ladder for nu_n < numax, Sigma_loc beyond, negative nu by conjugation
__global__ void k_g_ladder_full(int nq, int nf, int fft_lo, int numax, double beta, const double* mu_dev,
                                const double* eps, const double2* sigma, const double2* sigma_loc, double2* G) {
    const double mu = mu_dev[0];
    const int L = fft_lo + nf - 1;    // last index
    const size_t total = (size_t)nq * nf;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int q = (int)(e % nq), f = (int)(e / nq);
        const int vn = fft_lo + f;
        double2 g;
        if (vn >= 0) {
            const double2 s = vn < numax ? sigma[(size_t)vn * nq + q] : sigma_loc[vn];
            g = g_at(mu, eps[q], s, vn, beta);
        } else {
            // G_new[:, first:-1] = conj(G_new[:, last-1:-1:0])  (GFTools.jl:183-184)
            const int src = (L - 1) - (vn - fft_lo);
            const double2 s = src < numax ? sigma[(size_t)src * nq + q] : sigma_loc[src];
            g = cconj(g_at(mu, eps[q], s, src, beta));
        }
        G[e] = g;
    }
}

__global__ void k_fill_tail(int nq, int numax, double beta, double tnum, double2* out, int out_ld) {
    const int total = nq * numax;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        const int q = e % nq, nn = e / nq;
        const double w = (2.0 * nn + 1.0) * M_PI / beta;
        out[(size_t)nn * out_ld + q] = make_double2(0.0, -tnum / w);
    }
}

// lambda_m right-hand side and bounds on the stream (no host round trip):
// out[0] = 2 imp_density - sum_kω(chi_d) is formed inside k_lambda_m from these pieces.

SumArgs sum_args(const ldga_ctx* ctx) {
    SumArgs a;
    a.nq = ctx->Nq; a.nw = ctx->Nw; a.n_iw = ctx->sp.n_iw;
    a.beta = ctx->mp.beta; a.c2 = ctx->mp.Ekin_DMFT; a.inv_nk = 1.0 / (double)ctx->Nk;
    return a;
}

GArgs g_args(const ldga_ctx* ctx, int numax, double shell) {
    GArgs a;
    a.nq = ctx->Nq; a.numax = numax; a.beta = ctx->mp.beta; a.U = ctx->mp.U; a.n = ctx->mp.n;
    a.inv_nk = 1.0 / (double)ctx->Nk;
    a.shell = shell;
    return a;
}

}  // namespace

// trigamma psi_1(x) for x > 0: recurrence up to x >= 8, then the asymptotic series
// psi_1(x) ~ 1/x + 1/(2x^2) + sum_k B_2k / x^(2k+1)  (Abramowitz & Stegun 6.4.12)
double host_trigamma(double x) {
    double acc = 0.0;
    while (x < 8.0) { acc += 1.0 / (x * x); x += 1.0; }
    const double x2 = 1.0 / (x * x);
    const double series = 1.0 / x + x2 / 2.0 +
        (1.0 / 6.0 - x2 * (1.0 / 30.0 - x2 * (1.0 / 42.0 - x2 * (1.0 / 30.0 - x2 * (5.0 / 66.0 - x2 * (691.0 / 2730.0 - x2 * (7.0 / 6.0))))))) / (x * x * x);
    return acc + series;
}

// G_shell_sum (GFTools.jl:281-283): psi_1(1/2 - N) = pi^2 - psi_1(N + 1/2) by the reflection formula.
double host_G_shell_sum(int N, double beta) {
    const double a = host_trigamma(N + 0.5);
    const double b = M_PI * M_PI - a;
    return (a - b) * beta / (4.0 * M_PI * M_PI) + beta / 4.0;
}

int launch_F_from_chi(ldga_ctx* ctx, const double2* d_chi_loc, const double2* d_gimp, int n_gimp) {
    (void)n_gimp;
    StageTimer st_(ctx, LDGA_STAGE_LAMBDA0);
    k_F_from_chi<<<256, 256, 0, ctx->stream>>>(ctx->Nnu, ctx->Nw, ctx->sp.n_iv, ctx->sp.n_iw, ctx->sp.shift,
                                              ctx->mp.beta, d_chi_loc, d_gimp, ctx->d_F);
    LDGA_LAUNCHED(ctx, "k_F_from_chi");
    return LDGA_OK;
}

// ---------------------------------------------------------------------------------------------
// Gradient of E_pot,1 = calc_E(G_ladder(Σ, μ(Σ)), Σ, μ) with respect to Σ_ladder [Nq, numax]
// (thermodynamics.jl:142-168, GFTools.jl:154-186), μ following the filling condition
// f(μ, Σ) = 2(2 Re Σ_n G_k(n)/β + 1/2 + μ s)/(1 + U s) - n = 0 (s = G_shell_sum):
//   G = 1/(iν_n + μ - ε - Σ),  A = (2/(β N_k)) kMult conj(G (1 + Σ G))          (∂E/∂Σ at fixed μ)
//   ∂E/∂μ = (1/(β N_k)) Σ_q kMult [2 Σ_n (Re(-G² Σ) - U n/2 / ν_n²) + β² U n/8]
//   ∂f/∂μ = 2 (2 Re Σ_n (1/N_k) Σ_q kMult (-G²)/β + s)/(1 + U s),
//   B = 4/(β (1 + U s)) kMult/N_k conj(G²)                                      (∂f/∂Σ)
//   out = A - (∂E/∂μ / ∂f/∂μ) B.   One CTA: two fixed-order reductions, then the elementwise pass.
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_epot_vjp(int nq, int numax, double beta, double U, double nfill, double mu,
                                                   double shell, double inv_nk, const double* __restrict__ kmult,
                                                   const double* __restrict__ eps, const double2* __restrict__ sigma,
                                                   double2* __restrict__ out) {
    __shared__ double red[2][32];
    const double hartree = nfill * U / 2.0;
    double dEdmu = 0.0, dfdmu = 0.0;
    const int total = nq * numax;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
        const int q = e % nq, n = e / nq;
        const double vn = (2.0 * n + 1.0) * M_PI / beta;
        const double2 s = sigma[e];
        const double2 g = cinv(make_double2(mu - eps[q] - s.x, vn - s.y));
        const double2 g2 = cmul(g, g);
        const double2 g2s = cmul(g2, s);
        dEdmu += kmult[q] * (2.0 * (-g2s.x - hartree / (vn * vn)));
        dfdmu += kmult[q] * (-g2.x);
    }
    for (int o = 16; o > 0; o >>= 1) {
        dEdmu += __shfl_down_sync(0xffffffffu, dEdmu, o);
        dfdmu += __shfl_down_sync(0xffffffffu, dfdmu, o);
    }
    if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = dEdmu; red[1][threadIdx.x >> 5] = dfdmu; }
    __syncthreads();
    double sE = 0.0, sf = 0.0, km = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) { sE += red[0][i]; sf += red[1][i]; }
    for (int q = 0; q < nq; ++q) km += kmult[q];                                // N_k
    // the tail constant β² U n/8 per k point, weighted by kMult: Σ_q kMult = N_k
    const double dE = (sE + km * beta * beta * hartree / 4.0) * inv_nk / beta;
    const double df = 2.0 * (2.0 * sf * inv_nk / beta + shell) / (1.0 + U * shell);
    const double r = dE / df;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
        const int q = e % nq, n = e / nq;
        const double vn = (2.0 * n + 1.0) * M_PI / beta;
        const double2 s = sigma[e];
        const double2 g = cinv(make_double2(mu - eps[q] - s.x, vn - s.y));
        const double2 a = cscale(cconj(cmul(g, cadd(make_double2(1.0, 0.0), cmul(s, g)))), 2.0 * kmult[q] * inv_nk / beta);
        const double2 b = cscale(cconj(cmul(g, g)), 4.0 / (beta * (1.0 + U * shell)) * kmult[q] * inv_nk);
        out[e] = make_double2(a.x - r * b.x, a.y - r * b.y);
    }
}

int launch_epot_vjp(ldga_ctx* ctx, int numax, double mu, const double2* sigma, double2* out) {
    k_epot_vjp<<<1, 1024, 0, ctx->stream>>>(ctx->Nq, numax, ctx->mp.beta, ctx->mp.U, ctx->mp.n, mu,
                                            host_G_shell_sum(numax + 1, ctx->mp.beta), 1.0 / (double)ctx->Nk,
                                            ctx->d_kmult, ctx->d_eps, sigma, out);
    LDGA_LAUNCHED(ctx, "k_epot_vjp");
    return LDGA_OK;
}

int launch_lambda0_vjp(ldga_ctx* ctx, const double2* l0_bar, double2* chi0_bar) {
    double2* colF = reinterpret_cast<double2*>(ctx->d_red + 64);
    k_colsum_F<<<std::min(4 * 148, (ctx->Nnu * ctx->Nw + 7) / 8), 256, 0, ctx->stream>>>(ctx->Nnu, ctx->Nw, ctx->d_F, colF);
    LDGA_LAUNCHED(ctx, "k_colsum_F");
    k_lambda0_vjp<<<4 * 148, 256, 0, ctx->stream>>>(ctx->Nq, ctx->Nnu, ctx->Nw, 1.0 / (ctx->mp.beta * ctx->mp.beta),
                                                    colF, l0_bar, chi0_bar);
    LDGA_LAUNCHED(ctx, "k_lambda0_vjp");
    return LDGA_OK;
}

int launch_lambda0(ldga_ctx* ctx) {
    double2* colF = reinterpret_cast<double2*>(ctx->d_red + 64);
    StageTimer st_(ctx, LDGA_STAGE_LAMBDA0);
    k_colsum_F<<<std::min(4 * 148, (ctx->Nnu * ctx->Nw + 7) / 8), 256, 0, ctx->stream>>>(ctx->Nnu, ctx->Nw, ctx->d_F, colF);
    LDGA_LAUNCHED(ctx, "k_colsum_F");
    // an ω shard: the same arrays advanced to w_lo (ω is their slowest index)
    const size_t w0 = (size_t)ctx->w_lo, nqv = (size_t)ctx->Nq * ctx->Nnu;
    k_lambda0<<<4 * 148, 256, 0, ctx->stream>>>(ctx->Nq, ctx->Nnu, shard_nw(ctx), 1.0 / (ctx->mp.beta * ctx->mp.beta),
                                                ctx->d_chi0 + w0 * nqv, colF + w0 * ctx->Nnu,
                                                ctx->d_lambda0 + w0 * nqv);
    LDGA_LAUNCHED(ctx, "k_lambda0");
    return LDGA_OK;
}

// mode 0: chi_lambda, 1: dchi_lambda, 2: sum_ωk order.  lam_dev (may be null) is added to lam.
int launch_sum_kw(ldga_ctx* ctx, int channel, double lam, int mode, double* d_out, const double* lam_dev) {
    StageTimer st_(ctx, LDGA_STAGE_SUMS);
    k_sum_kw<<<kCluster, kClThreads, 0, ctx->stream>>>(sum_args(ctx), ctx->d_chi[channel], ctx->d_kmult, lam, lam_dev,
                                                       mode, d_out);
    LDGA_LAUNCHED(ctx, "k_sum_kw");
    return LDGA_OK;
}

namespace {

// sum_kω(χ_m^λm) -> out_m[0] and sum_kω(χ_d^λd) -> out_d[0] in one launch: the same per-thread
// order and reduction as two k_sum_kw (mode 0) launches, so the values are the same bit for bit
__global__ void __cluster_dims__(kCluster, 1, 1) __launch_bounds__(kClThreads)
k_sum_kw2(SumArgs a, const double* __restrict__ chi_m, const double* __restrict__ chi_d,
          const double* __restrict__ kmult, double lam_m, double lam_d, double* out_m, double* out_d) {
    __shared__ ClRed<2> cr;
    int parity = 0;
    double v[2] = {0.0, 0.0};
    const int total = a.nq * a.nw;
    for (int e = cl_tid(); e < total; e += cl_nth()) {
        const double km = kmult[e % a.nq];
        const double xm = chi_m[e], xd = chi_d[e];
        v[0] = fma(km, lam_m != 0.0 ? xm / (lam_m * xm + 1.0) : xm, v[0]);
        v[1] = fma(km, lam_d != 0.0 ? xd / (lam_d * xd + 1.0) : xd, v[1]);
    }
    cluster_sum<2>(v, cr, parity);
    if (cl_tid() == 0) {
        out_m[0] = finish_kw(a, v[0]);
        out_d[0] = finish_kw(a, v[1]);
    }
    cg::this_cluster().sync();
}

}  // namespace

int launch_sum_kw2(ldga_ctx* ctx, double lam_m, double lam_d, double* d_out_m, double* d_out_d) {
    StageTimer st_(ctx, LDGA_STAGE_SUMS);
    k_sum_kw2<<<kCluster, kClThreads, 0, ctx->stream>>>(sum_args(ctx), ctx->d_chi[LDGA_CH_M], ctx->d_chi[LDGA_CH_D],
                                                        ctx->d_kmult, lam_m, lam_d, d_out_m, d_out_d);
    LDGA_LAUNCHED(ctx, "k_sum_kw2");
    return LDGA_OK;
}

// update_tail! (DataTypes.jl:315-345) of the c2/(i w)^2 tail: chi[:, w] += Re((c2_new - c2_old)/(i w_m)^2)
// = -(c2_new - c2_old)/w_m^2 for every w_m = 2 pi m / beta != 0.
__global__ void k_chi_tail_shift(int nq, int nw, int n_iw, double beta, double dc2, double* __restrict__ chi) {
    const size_t total = (size_t)nq * nw;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int m = (int)(e / nq) - n_iw;
        if (m == 0) continue;
        const double wm = 2.0 * M_PI * (double)m / beta;
        chi[e] -= dc2 / (wm * wm);
    }
}

int launch_chi_tail_shift(ldga_ctx* ctx, int channel, double dc2) {
    k_chi_tail_shift<<<2 * 148, 256, 0, ctx->stream>>>(ctx->Nq, ctx->Nw, ctx->sp.n_iw, ctx->mp.beta, dc2,
                                                      ctx->d_chi[channel]);
    LDGA_LAUNCHED(ctx, "k_chi_tail_shift");
    return LDGA_OK;
}

using NewtonKern = void (*)(SumArgs, const double*, const double*, double, const double*, int, double*, int, double,
                           double*, const double*, double*, double*);

// Register-resident elements per thread K for `per` (q, ω) terms per thread; K = 0 streams them.
template <bool AS, int CL>
NewtonKern pick_newton(int per) {
    return per <= 2 ? k_lambda_m<2, AS, CL> : per <= 4 ? k_lambda_m<4, AS, CL> : per <= 6 ? k_lambda_m<6, AS, CL>
         : per <= 8 ? k_lambda_m<8, AS, CL> : per <= 10 ? k_lambda_m<10, AS, CL> : per <= 12 ? k_lambda_m<12, AS, CL>
         : per <= 16 ? k_lambda_m<16, AS, CL> : per <= 20 ? k_lambda_m<20, AS, CL> : per <= 24 ? k_lambda_m<24, AS, CL>
         : k_lambda_m<0, AS, CL>;
}

using MuKern = void (*)(GArgs, const double*, const double*, const double2*, int, double, const double*, double*);

template <int CL, int NT>
MuKern pick_mu(int per) {
    return per <= 2 ? k_mu_fit_energy<2, CL, NT> : per <= 4 ? k_mu_fit_energy<4, CL, NT>
         : per <= 6 ? k_mu_fit_energy<6, CL, NT> : per <= 8 ? k_mu_fit_energy<8, CL, NT>
         : k_mu_fit_energy<0, CL, NT>;
}

int launch_lambda_min(ldga_ctx* ctx, int channel, double* d_out) {
    const int w0 = (ctx->Nw + 1) / 2 - 1;   // ω0_index = ceil(Nw/2), 1-based
    StageTimer st_(ctx, LDGA_STAGE_SUMS);
    k_lambda_min<<<1, 1024, 0, ctx->stream>>>(ctx->Nq, w0, ctx->d_chi[channel], d_out);
    LDGA_LAUNCHED(ctx, "k_lambda_min");
    return LDGA_OK;
}

// lambda_m Newton: rhs = rhs_const - *rhs_sub_dev (if given); d_out[0] = lambda, d_out[1] = iterations;
// d_out[2] receives lambda_min; d_out[3..4] the periodic-trajectory skip (iteration, period).
int launch_lambda_m(ldga_ctx* ctx, double rhs_const, const double* rhs_sub_dev, double* d_out, int nsteps,
                    double atol, double* sum_d_out, double* sum_m_out) {
    const int w0 = (ctx->Nw + 1) / 2 - 1;   // ω0_index = ceil(Nw/2), 1-based; get_λ_min's column
    StageTimer st_(ctx, LDGA_STAGE_LAMBDA_NEWTON);
    const SumArgs sa = sum_args(ctx);
    const int cl = ctx->newton_cluster;
    const int per = (sa.nq * sa.nw + cl * kNewtonThreads - 1) / (cl * kNewtonThreads);
    const NewtonKern kern = cl == 16 ? pick_newton<true, 16>(per)
                          : ctx->newton_async ? pick_newton<true, kCluster>(per) : pick_newton<false, kCluster>(per);
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)cl;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3((unsigned)cl);
    cfg.blockDim = dim3(kNewtonThreads);
    cfg.stream = ctx->stream;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, kern, sa, (const double*)ctx->d_chi[LDGA_CH_M],
                                             (const double*)ctx->d_kmult, rhs_const, rhs_sub_dev,
                                             w0, d_out + 2, nsteps, atol, d_out,
                                             (const double*)(sum_d_out ? ctx->d_chi[LDGA_CH_D] : nullptr),
                                             sum_d_out, sum_m_out);
    if (e != cudaSuccess) return ctx_fail(ctx, LDGA_ERR_CUDA, std::string("k_lambda_m launch: ") + cudaGetErrorString(e));
    LDGA_LAUNCHED(ctx, "k_lambda_m");
    return LDGA_OK;
}

// Cluster size of the λm Newton on the current device: 16 CTAs where the GPU can co-schedule a
// non-portable 16-CTA cluster of this kernel, else the portable 8.  The barrier form
// (async = false) keeps 8.  Called by ldga_create with the handle's device current; the
// environment variable LDGA_NEWTON_CLUSTER=8 keeps 8 for comparison.
int newton_cluster_size(bool async) {
    if (!async) return kCluster;
    if (const char* s = std::getenv("LDGA_NEWTON_CLUSTER"))
        if (std::atoi(s) == kCluster) return kCluster;
    const NewtonKern all16[] = {k_lambda_m<2, true, 16>, k_lambda_m<4, true, 16>, k_lambda_m<6, true, 16>,
                                k_lambda_m<8, true, 16>, k_lambda_m<10, true, 16>, k_lambda_m<12, true, 16>,
                                k_lambda_m<16, true, 16>, k_lambda_m<20, true, 16>, k_lambda_m<24, true, 16>,
                                k_lambda_m<0, true, 16>};
    for (NewtonKern k : all16)
        if (cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
            cudaGetLastError();
            return kCluster;
        }
    const MuKern mu16[] = {k_mu_fit_energy<2, 16, kNewtonThreads>, k_mu_fit_energy<4, 16, kNewtonThreads>,
                           k_mu_fit_energy<6, 16, kNewtonThreads>, k_mu_fit_energy<8, 16, kNewtonThreads>,
                           k_mu_fit_energy<0, 16, kNewtonThreads>};
    for (MuKern k : mu16)
        if (cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
            cudaGetLastError();
            return kCluster;
        }
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = 16;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(16);
    cfg.blockDim = dim3(kNewtonThreads);
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int n = 0;
    for (NewtonKern k : all16)
        if (cudaOccupancyMaxActiveClusters(&n, k, &cfg) != cudaSuccess || n < 1) {
            cudaGetLastError();
            return kCluster;
        }
    for (MuKern k : mu16)
        if (cudaOccupancyMaxActiveClusters(&n, k, &cfg) != cudaSuccess || n < 1) {
            cudaGetLastError();
            return kCluster;
        }
    return 16;
}

int launch_g_ladder(ldga_ctx* ctx, int numax, int fix_n, double mu_in, double* d_out, const double* mu_dev) {
    GArgs a = g_args(ctx, numax, host_G_shell_sum(numax + 1, ctx->mp.beta));
    StageTimer st_(ctx, LDGA_STAGE_GLADDER);
    const int cl = ctx->newton_cluster, nt = cl == 16 ? kNewtonThreads : kClThreads;
    const int per = (a.nq * a.numax + cl * nt - 1) / (cl * nt);
    const MuKern kern = cl == 16 ? pick_mu<16, kNewtonThreads>(per) : pick_mu<kCluster, kClThreads>(per);
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)cl;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3((unsigned)cl);
    cfg.blockDim = dim3((unsigned)nt);
    cfg.stream = ctx->stream;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, kern, a, (const double*)ctx->d_kmult, (const double*)ctx->d_eps,
                                             (const double2*)ctx->d_sigma, fix_n, mu_in, mu_dev, d_out);
    if (e != cudaSuccess)
        return ctx_fail(ctx, LDGA_ERR_CUDA, std::string("k_mu_fit_energy launch: ") + cudaGetErrorString(e));
    LDGA_LAUNCHED(ctx, "k_mu_fit_energy");
    return LDGA_OK;
}

int launch_calc_E(ldga_ctx* ctx, const double2* G, int ldg, const double2* sigma, int numax, double mu,
                  double* d_out) {
    GArgs a = g_args(ctx, numax, 0.0);
    StageTimer st_(ctx, LDGA_STAGE_GLADDER);
    k_calc_E<<<kCluster, kClThreads, 0, ctx->stream>>>(a, ctx->d_kmult, ctx->d_eps, G, ldg, sigma, mu, d_out);
    LDGA_LAUNCHED(ctx, "k_calc_E");
    return LDGA_OK;
}

// mu_dev: device scalar with the chemical potential (e.g. the output of k_mu_fit_energy)
int launch_g_ladder_full(ldga_ctx* ctx, int numax, const double* mu_dev) {
    StageTimer st_(ctx, LDGA_STAGE_GLADDER);
    k_g_ladder_full<<<4 * 148, 256, 0, ctx->stream>>>(ctx->Nq, ctx->Nf, ctx->fft_lo, numax, ctx->mp.beta, mu_dev,
                                                      ctx->d_eps, ctx->d_sigma, ctx->d_sigma_loc, ctx->d_gladder);
    LDGA_LAUNCHED(ctx, "k_g_ladder_full");
    return LDGA_OK;
}

// ---------------------------------------------------------------------------------------------
// Allocation-free lambda_0 (ldga_lambda0_noalloc).
//
// Its one piece of scratch, the column sums colF[nu', w] = sum_nu F[nu, nu', w], lives in this
// file-scope device array instead of memory from cudaMalloc.  Every GPU that loads the library holds
// the array (LDGA_NOALLOC_MAX_COLS complex doubles, 512 KiB) until the process exits.  All calls share
// it: the column-sum kernel writes every entry the lambda_0 kernel reads, so nothing needs clearing,
// but two calls that run at the same time on one GPU (different streams, or host threads) race on it.
// ---------------------------------------------------------------------------------------------
#define LDGA_NOALLOC_MAX_COLS 32768
static __device__ __align__(256) double2 g_noalloc_colF[LDGA_NOALLOC_MAX_COLS];

namespace {
// Device address of g_noalloc_colF per device.  In host code the symbol's name is only a host-side
// stand-in; cudaGetSymbolAddress, called with the device current, gives the address a kernel can use.
double2* noalloc_colF(int device, cudaError_t* err) {
    static double2* addr[64] = {nullptr};
    static std::mutex mu;
    if (device < 0 || device >= 64) { *err = cudaErrorInvalidDevice; return nullptr; }
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[device]) {
        double2* p = nullptr;
        *err = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_noalloc_colF);
        if (*err != cudaSuccess) return nullptr;
        addr[device] = p;
    }
    *err = cudaSuccess;
    return addr[device];
}

// Device (or managed) memory that belongs to `device`: a pointer into another GPU's memory would be
// read as peer memory by the kernels, so it is refused like host memory.
bool is_device_ptr(const void* p, int device) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) { cudaGetLastError(); return false; }
    if (a.type == cudaMemoryTypeManaged) return true;
    return a.type == cudaMemoryTypeDevice && a.device == device;
}
}  // namespace

extern "C" int ldga_lambda0_noalloc(const double* chi0, const double* F, int32_t nq, int32_t nnu, int32_t nw,
                                    double beta, double* lambda0_out, void* stream) {
    if (!chi0 || !F || !lambda0_out) return ctx_fail(nullptr, LDGA_ERR_ARG, "ldga_lambda0_noalloc: null argument");
    if (nq < 1 || nnu < 1 || nw < 1) return ctx_fail(nullptr, LDGA_ERR_ARG, "ldga_lambda0_noalloc: sizes must be positive");
    if ((long)nnu * nw > LDGA_NOALLOC_MAX_COLS)
        return ctx_fail(nullptr, LDGA_ERR_ARG,
                        "ldga_lambda0_noalloc: Nnu*Nw = " + std::to_string((long)nnu * nw) +
                            " exceeds the built-in scratch of " + std::to_string(LDGA_NOALLOC_MAX_COLS) +
                            " (nu', w) columns");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return ctx_fail(nullptr, LDGA_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (!is_device_ptr(chi0, dev) || !is_device_ptr(F, dev) || !is_device_ptr(lambda0_out, dev))
        return ctx_fail(nullptr, LDGA_ERR_ARG,
                        "ldga_lambda0_noalloc: chi0, F and lambda0_out must be device memory of the current device");
    double2* colF = noalloc_colF(dev, &e);
    if (!colF) return ctx_fail(nullptr, LDGA_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_colsum_F<<<std::min(4 * 148, (nnu * nw + 7) / 8), 256, 0, s>>>(nnu, nw, reinterpret_cast<const double2*>(F), colF);
    k_lambda0<<<4 * 148, 256, 0, s>>>(nq, nnu, nw, 1.0 / (beta * beta), reinterpret_cast<const double2*>(chi0), colF,
                                      reinterpret_cast<double2*>(lambda0_out));
    e = cudaGetLastError();
    if (e != cudaSuccess) return ctx_fail(nullptr, LDGA_ERR_CUDA, std::string("ldga_lambda0_noalloc launch: ") + cudaGetErrorString(e));
    return LDGA_OK;
}

int launch_fill_tail(ldga_ctx* ctx, int numax, double tnum, double2* out, int out_ld) {
    k_fill_tail<<<64, 256, 0, ctx->stream>>>(ctx->Nq, numax, ctx->mp.beta, tnum, out, out_ld);
    LDGA_LAUNCHED(ctx, "k_fill_tail");
    return LDGA_OK;
}
