// k-space kernels: lattice G and its transform (setup), the bubble chi0, and the equation of motion.
// All of them are built on the symmetry-reduced transform of transform.cuh; one CTA processes a
// batch of independent (nu, w) vectors entirely in shared memory.
#include <cmath>

#include "transform.cuh"

using namespace ldga;

namespace {

constexpr int kThreads = 256;
// the CUDA-core transform kernels of the G setup, bubble and EoM: 16 warps per CTA where a thread's
// column (M complex values in registers) fits 128 registers, so one CTA per SM still has warps to hide
// the shared-memory and FMA latencies; 8 warps above
template <int M, bool TC>
constexpr int kThr = (!TC && M <= 17) ? 512 : kThreads;
constexpr size_t kSmemBudget = 200 * 1024;
// the tensor-path transform kernels run two CTAs per SM: half the shared memory each
constexpr size_t kSmemBudgetTC = 110 * 1024;

template <int DIM, int M>
int pairs_per_cta(int total, size_t budget = kSmemBudget) {
    using S = TransformSmem<DIM, M>;
    const size_t per = (size_t)(S::BUF_A + S::BUF_B) * sizeof(double2);
    int np = (int)(budget / per);
    if (np > 16) np = 16;
    // batch vectors into a CTA only when there are more vectors than SMs: a short list (the EoM
    // inverse's numax vectors) runs one vector per CTA on as many SMs
    const int spread = (total + 147) / 148;
    if (np > spread) np = spread;
    if (np < 1) np = 1;
    if (np > total) np = total;
    return np;
}

template <int DIM, int M>
size_t smem_bytes(int np) {
    using S = TransformSmem<DIM, M>;
    return (size_t)np * (S::BUF_A + S::BUF_B) * sizeof(double2);
}

template <int M>
TMat<M> make_T(const ldga_ctx* ctx) {
    TMat<M> T;
    for (int i = 0; i < M * M; ++i) T.t[i] = ctx->Tmat[i];
    return T;
}

// ---------------------------------------------------------------------------------------------
// a1: G(k, nu) for nu in fft_range and Ghat = S(G)
// ---------------------------------------------------------------------------------------------
template <int DIM, int M, bool TC>
__global__ void __launch_bounds__((kThr<M, TC>), TC ? 2 : 1) k_gloc_transform(
    const TMat<M> T, int nf, int fft_lo, double beta, double mu, const double* __restrict__ eps,
    const double2* __restrict__ sigma_loc, int n_sigma, double2* __restrict__ gloc, int from_sigma,
    double2* __restrict__ ghat, int np_max) {
    using S = TransformSmem<DIM, M>;
    constexpr int NQ = S::NQ;
    extern __shared__ double2 smem[];
    const int p0 = blockIdx.x * np_max;
    const int np = min(np_max, nf - p0);
    double2* bufA = smem;
    double2* bufB = smem + np_max * S::BUF_A;
    for (int it = threadIdx.x; it < np * NQ; it += blockDim.x) {
        const int p = it / NQ, q = it - p * NQ;
        const int f = p0 + p;
        double2 g;
        if (from_sigma) {
            const int vn = fft_lo + f;
            const double2 s = vn < 0 ? cconj(sigma_loc[-vn - 1]) : sigma_loc[vn];
            const double2 z = make_double2(mu - eps[q] - s.x, (2.0 * vn + 1.0) * M_PI / beta - s.y);
            g = cinv(z);
            gloc[(size_t)f * NQ + q] = g;
        } else {
            g = gloc[(size_t)f * NQ + q];
        }
        bufA[p * NQ + q] = g;
    }
    __syncthreads();
    sym_transform_any<DIM, M, TC>(np, bufA, bufB, T, [&](int p, int q, double2 v) {
        ghat[(size_t)(p0 + p) * NQ + q] = v;
    });
}

// ---------------------------------------------------------------------------------------------
// a2: chi0[q, nu, w] = -beta/N_k^2 S(Ghat(nu) Ghat(nu+w))(q)
// G(k, -nu) = conj(G(k, nu)) (nu_n -> nu_{-n-1}) and G is even in k, so
//   chi0(q, nu'', w) = conj(chi0(q, nu, w)),  nu'' = -nu - w - 1,
// and a pair whose partner lies in the box is computed once: `pairs` lists the representatives
// (pair index vi + Nnu wi, partner's index or -1), built on the host with the handle.
// ---------------------------------------------------------------------------------------------
template <int DIM, int M, bool TC>
__global__ void __launch_bounds__((kThr<M, TC>), TC ? 2 : 1) k_bubble(
    const TMat<M> T, int nnu, int nw, int n_iv, int n_iw, int shift, int fft_lo, double scale,
    const double2* __restrict__ ghat, const int2* __restrict__ pairs, int total, double2* __restrict__ chi0, int np_max) {
    using S = TransformSmem<DIM, M>;
    constexpr int NQ = S::NQ;
    extern __shared__ double2 smem[];
    const int p0 = blockIdx.x * np_max;
    const int np = min(np_max, total - p0);
    double2* bufA = smem;
    double2* bufB = smem + np_max * S::BUF_A;
    for (int it = threadIdx.x; it < np * NQ; it += blockDim.x) {
        const int p = it / NQ, q = it - p * NQ;
        const int pi = pairs[p0 + p].x;
        const int wi = pi / nnu, vi = pi - wi * nnu;
        const int wn = wi - n_iw;
        const int vn = (vi - n_iv) - shift * (wn / 2);    // C division truncates like trunc(Int, .)
        const double2 a = ghat[(size_t)(vn - fft_lo) * NQ + q];
        const double2 b = ghat[(size_t)(vn + wn - fft_lo) * NQ + q];
        bufA[p * NQ + q] = cmul(a, b);
    }
    __syncthreads();
    sym_transform_any<DIM, M, TC>(np, bufA, bufB, T, [&](int p, int q, double2 v) {
        const int2 pp = pairs[p0 + p];
        const double2 c = cscale(v, scale);
        chi0[(size_t)pp.x * NQ + q] = c;
        if (pp.y >= 0) chi0[(size_t)pp.y * NQ + q] = cconj(c);
    });
}

// ---------------------------------------------------------------------------------------------
// a9/a10: EoM.  Forward: for one nu_n and a chunk of w, K(q) = eom(...) -> S(K) * Ghat(nu+w),
// summed over the chunk in a fixed order -> partial[chunk][nu][q].  The inverse kernel then sums
// the chunks (fixed order), applies S, and adds 1/beta, the tail and the Hartree term.
// ---------------------------------------------------------------------------------------------
struct EomArgs {
    int nnu, nw, n_iv, n_iw, shift, fft_lo, numax, w_per_chunk;
    int w_begin = 0, w_end = 0;   // the ω range the forward kernel sums ([0, nw) without a shard)
    double U, lam_m, lam_d;
    const double* lam_m_dev;   // device scalars added to lam_m / lam_d (may be null)
    const double* lam_d_dev;
    int part;   // -1: full eom; 0..5: calc_Σ_parts contributions
};

__device__ __forceinline__ double chi_lam(double x, double lam) {
    return lam == 0.0 ? x : x / (lam * x + 1.0);
}

__device__ __forceinline__ double2 eom_value(const EomArgs& a, double2 gm, double2 gd, double xm, double xd,
                                             double2 l0) {
    const double U = a.U;
    switch (a.part) {
        case 0: {  // eom_χ_m = U*(γm*1.5*(U*χm))
            const double f = 1.5 * (U * xm);
            return make_double2(U * (gm.x * f), U * (gm.y * f));
        }
        case 1:    // eom_γ_m = U*(γm*1.5)
            return make_double2(U * (gm.x * 1.5), U * (gm.y * 1.5));
        case 2: {  // eom_χ_d = -U*(γd*0.5*(-U*χd))
            const double f = 0.5 * (-U * xd);
            return make_double2(-U * (gd.x * f), -U * (gd.y * f));
        }
        case 3:    // eom_γ_d = -U*(γd*0.5)
            return make_double2(-U * (gd.x * 0.5), -U * (gd.y * 0.5));
        case 4:    // eom_rest_01 = -U*1.0 + 0im
            return make_double2(-U * 1.0, 0.0);
        case 5:    // eom_rest = U*λ₀
            return make_double2(U * l0.x, U * l0.y);
        default: {
            // eom = U*(γm*1.5*(1+U*χm) - γd*0.5*(1-U*χd) - 1.5 + 0.5 + λ₀), left to right
            const double fm = 1.5 * (1.0 + U * xm);
            const double fd = 0.5 * (1.0 - U * xd);
            double re = gm.x * fm - gd.x * fd;
            double im = gm.y * fm - gd.y * fd;
            re = re - 1.5;
            re = re + 0.5;
            re = re + l0.x;
            im = im + l0.y;
            return make_double2(U * re, U * im);
        }
    }
}

template <int DIM, int M, bool TC>
__global__ void __launch_bounds__((kThr<M, TC>), TC ? 2 : 1) k_eom_forward(
    const TMat<M> T, const EomArgs a, const double2* __restrict__ ghat, const double* __restrict__ chi_m,
    const double2* __restrict__ gam_m, const double* __restrict__ chi_d, const double2* __restrict__ gam_d,
    const double2* __restrict__ lambda0, double2* __restrict__ partial) {
    using S = TransformSmem<DIM, M>;
    constexpr int NQ = S::NQ;
    extern __shared__ double2 smem[];
    const int np_max = a.w_per_chunk;
    const int chunk = blockIdx.x, nu_n = blockIdx.y;
    const int w0 = a.w_begin + chunk * np_max;
    const int np = min(np_max, a.w_end - w0);
    double2* bufA = smem;
    double2* bufB = smem + np_max * S::BUF_A;
    double2* outb = smem + np_max * (S::BUF_A + S::BUF_B);     // [np_max][NQ] products
    __shared__ int s_vi[16];
    if (threadIdx.x < np) {
        const int wi = w0 + threadIdx.x;
        const int wn = wi - a.n_iw;
        const int v0 = a.n_iv + a.shift * ((wi - a.n_iw) / 2);          // ν0Index_of_ωIndex - 1
        const int len = min(a.numax, 2 * a.n_iv - v0);
        s_vi[threadIdx.x] = (nu_n < len && v0 + nu_n >= 0) ? v0 + nu_n : -1;
        (void)wn;
    }
    __syncthreads();
    for (int it = threadIdx.x; it < np * NQ; it += blockDim.x) {
        const int p = it / NQ, q = it - p * NQ;
        const int wi = w0 + p;
        const int vi = s_vi[p];
        double2 K = make_double2(0.0, 0.0);
        if (vi >= 0) {
            const size_t iq = (size_t)q + (size_t)NQ * wi;
            const size_t iv = (size_t)q + (size_t)NQ * (vi + (size_t)a.nnu * wi);
            const double lm = a.lam_m + (a.lam_m_dev ? a.lam_m_dev[0] : 0.0);
            const double ld = a.lam_d + (a.lam_d_dev ? a.lam_d_dev[0] : 0.0);
            const double xm = chi_lam(chi_m[iq], lm);
            const double xd = chi_lam(chi_d[iq], ld);
            K = eom_value(a, gam_m[iv], gam_d[iv], xm, xd, lambda0[iv]);
        }
        bufA[p * NQ + q] = K;
    }
    __syncthreads();
    sym_transform_any<DIM, M, TC>(np, bufA, bufB, T, [&](int p, int q, double2 v) {
        const int wi = w0 + p;
        const int wn = wi - a.n_iw;
        double2 r = make_double2(0.0, 0.0);
        if (s_vi[p] >= 0) r = cmul(v, ghat[(size_t)(nu_n + wn - a.fft_lo) * NQ + q]);
        outb[p * NQ + q] = r;
    });
    for (int q = threadIdx.x; q < NQ; q += blockDim.x) {
        double2 acc = make_double2(0.0, 0.0);
        for (int p = 0; p < np; ++p) acc = cadd(acc, outb[p * NQ + q]);
        partial[((size_t)chunk * a.numax + nu_n) * NQ + q] = acc;
    }
}

template <int DIM, int M, bool TC>
__global__ void __launch_bounds__((kThr<M, TC>), TC ? 2 : 1) k_eom_inverse(
    const TMat<M> T, int numax, int nchunk, double scale, double beta, double U, double hartree,
    const double* __restrict__ tail_sum, int tc, double chiloc_m_sum, const double2* __restrict__ partial,
    double2* __restrict__ out, int out_ld, int add_hartree, int np_max) {
    using S = TransformSmem<DIM, M>;
    constexpr int NQ = S::NQ;
    extern __shared__ double2 smem[];
    const int p0 = blockIdx.x * np_max;
    const int np = min(np_max, numax - p0);
    double2* bufA = smem;
    double2* bufB = smem + np_max * S::BUF_A;
    for (int it = threadIdx.x; it < np * NQ; it += blockDim.x) {
        const int p = it / NQ, q = it - p * NQ;
        const int nu = p0 + p;
        double2 acc = make_double2(0.0, 0.0);
        for (int c = 0; c < nchunk; ++c) acc = cadd(acc, partial[((size_t)c * numax + nu) * NQ + q]);
        bufA[p * NQ + q] = acc;
    }
    __syncthreads();
    // tail: (tc ? -U (sum_kω χm - χloc_m_sum) : 0) / (i ν_n), ν_n = (2n+1)π/β
    const double tnum = tc ? -U * (tail_sum[0] - chiloc_m_sum) : 0.0;
    sym_transform_any<DIM, M, TC>(np, bufA, bufB, T, [&](int p, int q, double2 v) {
        const int nu = p0 + p;
        const double w = (2.0 * nu + 1.0) * M_PI / beta;
        // tnum / (i w) = -i tnum / w
        double re = v.x * scale / beta + 0.0;
        double im = v.y * scale / beta - tnum / w;
        if (add_hartree) re += hartree;
        out[(size_t)nu * out_ld + q] = make_double2(re, im);
    });
}

// ---------------------------------------------------------------------------------------------
// Adjoint of the EoM (calc_Σ, ladderDGATools_singleCore.jl:49-136) for a real loss with upstream
// Sbar[q, n] = dL/dRe Σ + i dL/dIm Σ over the stored (irreducible) values.  The forward is
//   Σ(q, n) = (1/(β N_k²)) S( Σ_ω S(K(·, n, ω)) Ĝ(ν_n + ω) )(q) + tail(n) + Hartree,
// and on symmetric functions the transform satisfies Sᵀ = kMult S kMult⁻¹, so
//   K̄(q, n, ω) = kMult(q)/(β N_k²) S( conj(Ĝ(ν_n + ω)) · S(Sbar(·, n)/kMult) )(q),
// the same transform-product-transform shape as the bubble.  From K = eom(γm, γd, χm^λ, χd^λ, λ₀):
//   γ̄m = 1.5 U (1 + U χm^λ) K̄,  γ̄d = -0.5 U (1 - U χd^λ) K̄,  λ̄₀ = U K̄,
//   χ̄m^λ += Σ_n Re(conj(K̄) 1.5 U² γm),  χ̄d^λ += Σ_n Re(conj(K̄) 0.5 U² γd),
// plus, with the tail correction, χ̄m^λ(q, ω) += s̄ kMult(q)/(β N_k) with s̄ = U Σ Im(Sbar)/ν_n
// (the tail is -U(sum_kω χm^λ - χloc_m_sum)/(iν_n)), and finally χ̄ = χ̄^λ/(λχ + 1)².
// ---------------------------------------------------------------------------------------------
template <int DIM, int M>
__global__ void __launch_bounds__(kThreads) k_vjp_sbar(const TMat<M> T, int numax, const double* __restrict__ kmult,
                                                       const double2* __restrict__ sbar, double2* __restrict__ shat, int np_max) {
    using S = TransformSmem<DIM, M>;
    constexpr int NQ = S::NQ;
    extern __shared__ double2 smem[];
    const int p0 = blockIdx.x * np_max;
    const int np = min(np_max, numax - p0);
    double2* bufA = smem;
    double2* bufB = smem + np_max * S::BUF_A;
    for (int it = threadIdx.x; it < np * NQ; it += blockDim.x) {
        const int p = it / NQ, q = it - p * NQ;
        bufA[p * NQ + q] = cscale(sbar[(size_t)(p0 + p) * NQ + q], 1.0 / kmult[q]);
    }
    __syncthreads();
    sym_transform<DIM, M>(np, bufA, bufB, T, [&](int p, int q, double2 v) {
        shat[(size_t)(p0 + p) * NQ + q] = v;
    });
}

struct EomVjpArgs {
    int nnu, nw, n_iv, n_iw, shift, fft_lo, numax;
    double U, lam_m, lam_d, scale;   // scale = 1/(beta N_k^2)
};

template <int DIM, int M>
__global__ void __launch_bounds__(kThreads) k_eom_vjp(
    const TMat<M> T, const EomVjpArgs a, const double* __restrict__ kmult, const double2* __restrict__ ghat,
    const double2* __restrict__ shat, const double* __restrict__ chi_m, const double2* __restrict__ gam_m,
    const double* __restrict__ chi_d, const double2* __restrict__ gam_d, double2* __restrict__ gm_bar,
    double2* __restrict__ gd_bar, double2* __restrict__ l0_bar, double* __restrict__ cm, double* __restrict__ cd, int np_max) {
    using S = TransformSmem<DIM, M>;
    constexpr int NQ = S::NQ;
    extern __shared__ double2 smem[];
    const int total = a.numax * a.nw;
    const int p0 = blockIdx.x * np_max;
    const int np = min(np_max, total - p0);
    double2* bufA = smem;
    double2* bufB = smem + np_max * S::BUF_A;
    __shared__ int s_vi[16];
    if (threadIdx.x < np) {
        const int pi = p0 + threadIdx.x;
        const int wi = pi / a.numax, n = pi - wi * a.numax;
        const int v0 = a.n_iv + a.shift * ((wi - a.n_iw) / 2);          // ν0Index_of_ωIndex - 1
        const int len = min(a.numax, 2 * a.n_iv - v0);
        s_vi[threadIdx.x] = (n < len && v0 + n >= 0) ? v0 + n : -1;
    }
    __syncthreads();
    for (int it = threadIdx.x; it < np * NQ; it += blockDim.x) {
        const int p = it / NQ, q = it - p * NQ;
        const int pi = p0 + p;
        const int wi = pi / a.numax, n = pi - wi * a.numax;
        const int wn = wi - a.n_iw;
        double2 v = make_double2(0.0, 0.0);
        if (s_vi[p] >= 0) v = cmul(shat[(size_t)n * NQ + q], cconj(ghat[(size_t)(n + wn - a.fft_lo) * NQ + q]));
        bufA[p * NQ + q] = v;
    }
    __syncthreads();
    sym_transform<DIM, M>(np, bufA, bufB, T, [&](int p, int q, double2 v) {
        const int pi = p0 + p;
        const int wi = pi / a.numax, n = pi - wi * a.numax;
        const int vi = s_vi[p];
        const size_t cslot = (size_t)n * NQ * a.nw + (size_t)q + (size_t)NQ * wi;
        if (vi < 0) {
            cm[cslot] = 0.0;
            cd[cslot] = 0.0;
            return;
        }
        const double2 kb = cscale(v, kmult[q] * a.scale);
        const size_t iq = (size_t)q + (size_t)NQ * wi;
        const size_t iv = (size_t)q + (size_t)NQ * (vi + (size_t)a.nnu * wi);
        const double U = a.U;
        const double xm = chi_lam(chi_m[iq], a.lam_m), xd = chi_lam(chi_d[iq], a.lam_d);
        if (gm_bar) gm_bar[iv] = cscale(kb, 1.5 * U * (1.0 + U * xm));
        if (gd_bar) gd_bar[iv] = cscale(kb, -0.5 * U * (1.0 - U * xd));
        if (l0_bar) l0_bar[iv] = cscale(kb, U);
        const double2 gm = gam_m[iv], gd = gam_d[iv];
        cm[cslot] = 1.5 * U * U * (kb.x * gm.x + kb.y * gm.y);    // Re(conj(kb) gm) 1.5 U^2
        cd[cslot] = 0.5 * U * U * (kb.x * gd.x + kb.y * gd.y);
    });
}

// s̄ = U Σ_{q,n} Im(Sbar(q, n)) / ν_n, one CTA, fixed order
__global__ void __launch_bounds__(256) k_vjp_tail(int nq, int numax, double beta, double U,
                                                   const double2* __restrict__ sbar, double* __restrict__ out) {
    __shared__ double red[8];
    double acc = 0.0;
    for (int e = threadIdx.x; e < nq * numax; e += blockDim.x) {
        const int n = e / nq;
        acc += sbar[e].y / ((2.0 * n + 1.0) * M_PI / beta);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0.0;
        for (int i = 0; i < 8; ++i) r += red[i];
        out[0] = U * r;
    }
}

__global__ void __launch_bounds__(256) k_eom_vjp_chi(int nq, int nw, int numax, double lam_m, double lam_d, double tail_w,
                                                      const double* __restrict__ kmult, const double* __restrict__ sb_dev,
                                                      const double* __restrict__ chi_m, const double* __restrict__ chi_d,
                                                      const double* __restrict__ cm, const double* __restrict__ cd,
                                                      double* __restrict__ xm_bar, double* __restrict__ xd_bar) {
    const size_t n_qw = (size_t)nq * nw;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n_qw; e += (size_t)gridDim.x * blockDim.x) {
        const int q = (int)(e % nq);
        double am = 0.0, ad = 0.0;
        for (int n = 0; n < numax; ++n) {
            am += cm[(size_t)n * n_qw + e];
            ad += cd[(size_t)n * n_qw + e];
        }
        if (tail_w != 0.0) am += sb_dev[0] * kmult[q] * tail_w;
        const double fm = lam_m * chi_m[e] + 1.0, fd = lam_d * chi_d[e] + 1.0;
        if (xm_bar) xm_bar[e] = am / (fm * fm);
        if (xd_bar) xd_bar[e] = ad / (fd * fd);
    }
}

// ---------------------------------------------------------------------------------------------
// Adjoint of the lattice G (setup + bubble + the EoM's direct use of Ĝ) -> dL/dΣ_loc.
//   bubble: χ₀(ν, ω) = s_b S(Ĝ(ν) Ĝ(ν+ω)), s_b = -β/N_k²  ->  P̄ = s_b kMult S(χ̄₀/kMult),
//           Ĝ̄(ν) += conj(Ĝ(ν+ω)) P̄,  Ĝ̄(ν+ω) += conj(Ĝ(ν)) P̄          (k_bubble_vjp)
//   EoM:    Σ(n) = c S(Σ_ω K̂(n,ω) Ĝ(ν_n+ω)), K̂ = S(K), c = 1/(β N_k²)
//           ->  Ĝ̄(ν_n+ω) += c kMult Ŝ̄(n) conj(K̂(n,ω)),  Ŝ̄ = S(Σ̄/kMult)   (k_eom_gvjp)
// Each (ν, ω) term writes its contribution to its own scratch row; k_ghat_gather sums, per
// frequency of fft_range, the rows that touch it in a fixed (host-computed) order.  Then
// Ḡ = kMult S(Ĝ̄/kMult) (k_vjp_transform) and, from G = 1/(iν + μ - ε - Σ_loc),
//   Σ̄_loc(m) = Σ_q conj(G²) Ḡ over ν_m,  + Σ_q conj(Ḡ) G² over ν_{-m-1}   (k_sigma_loc_grad).
// ---------------------------------------------------------------------------------------------
template <int DIM, int M>
__global__ void __launch_bounds__(kThreads) k_bubble_vjp(
    const TMat<M> T, int nnu, int nw, int n_iv, int n_iw, int shift, int fft_lo, double sb,
    const double* __restrict__ kmult, const double2* __restrict__ ghat, const double2* __restrict__ chi0_bar,
    double2* __restrict__ rows, int np_max) {
    using S = TransformSmem<DIM, M>;
    constexpr int NQ = S::NQ;
    extern __shared__ double2 smem[];
    const int total = nnu * nw;
    const int p0 = blockIdx.x * np_max;
    const int np = min(np_max, total - p0);
    double2* bufA = smem;
    double2* bufB = smem + np_max * S::BUF_A;
    for (int it = threadIdx.x; it < np * NQ; it += blockDim.x) {
        const int p = it / NQ, q = it - p * NQ;
        bufA[p * NQ + q] = cscale(chi0_bar[(size_t)(p0 + p) * NQ + q], 1.0 / kmult[q]);
    }
    __syncthreads();
    sym_transform<DIM, M>(np, bufA, bufB, T, [&](int p, int q, double2 v) {
        const int pi = p0 + p;
        const int wi = pi / nnu, vi = pi - wi * nnu;
        const int wn = wi - n_iw;
        const int vn = (vi - n_iv) - shift * (wn / 2);
        const double2 pb = cscale(v, sb * kmult[q]);
        const double2 g1 = ghat[(size_t)(vn - fft_lo) * NQ + q], g2 = ghat[(size_t)(vn + wn - fft_lo) * NQ + q];
        rows[(size_t)(2 * pi) * NQ + q] = cmul(cconj(g2), pb);       // -> frequency vn
        rows[(size_t)(2 * pi + 1) * NQ + q] = cmul(cconj(g1), pb);   // -> frequency vn + wn
    });
}

template <int DIM, int M>
__global__ void __launch_bounds__(kThreads) k_eom_gvjp(
    const TMat<M> T, const EomArgs a, double c, const double* __restrict__ kmult, const double2* __restrict__ shat,
    const double* __restrict__ chi_m, const double2* __restrict__ gam_m, const double* __restrict__ chi_d,
    const double2* __restrict__ gam_d, const double2* __restrict__ lambda0, double2* __restrict__ rows, int np_max) {
    using S = TransformSmem<DIM, M>;
    constexpr int NQ = S::NQ;
    extern __shared__ double2 smem[];
    const int total = a.numax * a.nw;
    const int p0 = blockIdx.x * np_max;
    const int np = min(np_max, total - p0);
    double2* bufA = smem;
    double2* bufB = smem + np_max * S::BUF_A;
    __shared__ int s_vi[16];
    if (threadIdx.x < np) {
        const int pi = p0 + threadIdx.x;
        const int wi = pi / a.numax, n = pi - wi * a.numax;
        const int v0 = a.n_iv + a.shift * ((wi - a.n_iw) / 2);
        const int len = min(a.numax, 2 * a.n_iv - v0);
        s_vi[threadIdx.x] = (n < len && v0 + n >= 0) ? v0 + n : -1;
    }
    __syncthreads();
    for (int it = threadIdx.x; it < np * NQ; it += blockDim.x) {
        const int p = it / NQ, q = it - p * NQ;
        const int wi = (p0 + p) / a.numax;
        const int vi = s_vi[p];
        double2 K = make_double2(0.0, 0.0);
        if (vi >= 0) {
            const size_t iq = (size_t)q + (size_t)NQ * wi;
            const size_t iv = (size_t)q + (size_t)NQ * (vi + (size_t)a.nnu * wi);
            K = eom_value(a, gam_m[iv], gam_d[iv], chi_lam(chi_m[iq], a.lam_m), chi_lam(chi_d[iq], a.lam_d), lambda0[iv]);
        }
        bufA[p * NQ + q] = K;
    }
    __syncthreads();
    sym_transform<DIM, M>(np, bufA, bufB, T, [&](int p, int q, double2 v) {
        const int pi = p0 + p;
        const int n = pi - (pi / a.numax) * a.numax;
        double2 r = make_double2(0.0, 0.0);
        if (s_vi[p] >= 0) r = cmul(cscale(shat[(size_t)n * NQ + q], c * kmult[q]), cconj(v));
        rows[(size_t)pi * NQ + q] = r;
    });
}

// out(f) = (mul_kmult ? kMult : 1) S(in(f) / kMult) for nf vectors of the wedge
template <int DIM, int M>
__global__ void __launch_bounds__(kThreads) k_vjp_transform(const TMat<M> T, int nf, int mul_kmult,
                                                            const double* __restrict__ kmult,
                                                            const double2* __restrict__ in, double2* __restrict__ out, int np_max) {
    using S = TransformSmem<DIM, M>;
    constexpr int NQ = S::NQ;
    extern __shared__ double2 smem[];
    const int p0 = blockIdx.x * np_max;
    const int np = min(np_max, nf - p0);
    double2* bufA = smem;
    double2* bufB = smem + np_max * S::BUF_A;
    for (int it = threadIdx.x; it < np * NQ; it += blockDim.x) {
        const int p = it / NQ, q = it - p * NQ;
        bufA[p * NQ + q] = cscale(in[(size_t)(p0 + p) * NQ + q], 1.0 / kmult[q]);
    }
    __syncthreads();
    sym_transform<DIM, M>(np, bufA, bufB, T, [&](int p, int q, double2 v) {
        out[(size_t)(p0 + p) * NQ + q] = mul_kmult ? cscale(v, kmult[q]) : v;
    });
}

// Ĝ̄[f][q] = Σ_{j in list(f)} rows[idx[j]][q], CSR over the fft_range frequencies, fixed order
__global__ void __launch_bounds__(256) k_ghat_gather(int nf, int nq, const int32_t* __restrict__ start,
                                                      const int32_t* __restrict__ idx, const double2* __restrict__ rows,
                                                      double2* __restrict__ gbar) {
    const size_t n = (size_t)nf * nq;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int f = (int)(e / nq), q = (int)(e % nq);
        double2 acc = make_double2(0.0, 0.0);
        for (int j = start[f]; j < start[f + 1]; ++j) acc = cadd(acc, rows[(size_t)idx[j] * nq + q]);
        gbar[e] = acc;
    }
}

// Σ̄_loc(m), m = 0..n_sigma-1: one CTA per m, fixed-order block reduction over q
__global__ void __launch_bounds__(256) k_sigma_loc_grad(int nq, int nf, int fft_lo, int n_sigma,
                                                         const double2* __restrict__ gloc, const double2* __restrict__ gbar,
                                                         double2* __restrict__ out) {
    __shared__ double2 red[8];
    const int m = blockIdx.x;
    if (m >= n_sigma) return;
    double2 acc = make_double2(0.0, 0.0);
    const int fp = m - fft_lo, fn = -m - 1 - fft_lo;   // columns of ν_m and ν_{-m-1}
    for (int q = threadIdx.x; q < nq; q += blockDim.x) {
        if (fp >= 0 && fp < nf) {
            const double2 g = gloc[(size_t)fp * nq + q];
            acc = cadd(acc, cmul(cconj(cmul(g, g)), gbar[(size_t)fp * nq + q]));
        }
        if (fn >= 0 && fn < nf) {
            const double2 g = gloc[(size_t)fn * nq + q];
            acc = cadd(acc, cmul(cconj(gbar[(size_t)fn * nq + q]), cmul(g, g)));
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        acc.x += __shfl_down_sync(0xffffffffu, acc.x, o);
        acc.y += __shfl_down_sync(0xffffffffu, acc.y, o);
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double2 r = make_double2(0.0, 0.0);
        for (int i = 0; i < 8; ++i) r = cadd(r, red[i]);
        out[m] = r;
    }
}

// ---------------------------------------------------------------------------------------------
// host-side dispatch on (DIM, M)
// ---------------------------------------------------------------------------------------------
template <int DIM, int M>
int run_gloc(ldga_ctx* ctx, bool from_sigma) {
    const bool tc = ctx->transform_tc;
    const int np = pairs_per_cta<DIM, M>(ctx->Nf, tc ? kSmemBudgetTC : kSmemBudget);
    const size_t sm = smem_bytes<DIM, M>(np);
    auto kern = tc ? k_gloc_transform<DIM, M, true> : k_gloc_transform<DIM, M, false>;
    LDGA_CUDA(ctx, set_smem(ctx, kern, sm));
    dim3 grid((ctx->Nf + np - 1) / np);
    StageTimer st_(ctx, LDGA_STAGE_GLOC);
    kern<<<grid, tc ? kThr<M, true> : kThr<M, false>, sm, ctx->stream>>>(make_T<M>(ctx), ctx->Nf, ctx->fft_lo, ctx->mp.beta, ctx->mp.mu,
                                               ctx->d_eps, ctx->d_sigma_loc, ctx->n_sigma_loc, ctx->d_gloc,
                                               from_sigma ? 1 : 0, ctx->d_ghat, np);
    LDGA_LAUNCHED(ctx, "k_gloc_transform");
    return LDGA_OK;
}

template <int DIM, int M>
int run_bubble(ldga_ctx* ctx) {
    // an ω shard takes the pairs of its frequencies: a contiguous range of the ω-major list
    const int first = ctx->bub_pair_w_start[ctx->w_lo];
    const int total = ctx->bub_pair_w_start[ctx->w_hi] - first;
    if (total <= 0) return LDGA_OK;
    const bool tc = ctx->transform_tc;
    const int np = pairs_per_cta<DIM, M>(total, tc ? kSmemBudgetTC : kSmemBudget);
    const size_t sm = smem_bytes<DIM, M>(np);
    auto kern = tc ? k_bubble<DIM, M, true> : k_bubble<DIM, M, false>;
    LDGA_CUDA(ctx, set_smem(ctx, kern, sm));
    dim3 grid((total + np - 1) / np);
    const double scale = -ctx->mp.beta / ((double)ctx->Nk * (double)ctx->Nk);
    StageTimer st_(ctx, LDGA_STAGE_BUBBLE);
    kern<<<grid, tc ? kThr<M, true> : kThr<M, false>, sm, ctx->stream>>>(make_T<M>(ctx), ctx->Nnu, ctx->Nw, ctx->sp.n_iv, ctx->sp.n_iw,
                                               ctx->sp.shift, ctx->fft_lo, scale, ctx->d_ghat, ctx->d_bub_pairs + first,
                                               total, ctx->d_chi0, np);
    LDGA_LAUNCHED(ctx, "k_bubble");
    return LDGA_OK;
}

template <int DIM, int M>
int run_eom(ldga_ctx* ctx, int numax, double lam_m, double lam_d, const double* lm_dev, const double* ld_dev,
            int part, int& nchunk_out) {
    using S = TransformSmem<DIM, M>;
    const size_t per = (size_t)(S::BUF_A + S::BUF_B + S::NQ) * sizeof(double2);
    const bool tc = ctx->transform_tc;
    int wpc = (int)((tc ? kSmemBudgetTC : kSmemBudget) / per);
    if (wpc > 16) wpc = 16;
    if (wpc < 1) wpc = 1;
    // spread the w axis (the shard's range) over enough CTAs to fill the machine
    const int nws = shard_nw(ctx);
    const int target_ctas = 2 * 148;
    while (wpc > 1 && (long)numax * ((nws + wpc - 1) / wpc) < target_ctas) --wpc;
    const int nchunk = (nws + wpc - 1) / wpc;
    const size_t need = (size_t)nchunk * numax * ctx->Nq;
    if (need > ctx->partial_elems) {
        if (ctx->d_partial) cudaFree(ctx->d_partial);
        ctx->d_partial = nullptr;
        LDGA_CUDA(ctx, cudaMalloc(&ctx->d_partial, need * sizeof(double2)));
        ctx->partial_elems = need;
    }
    EomArgs a;
    a.nnu = ctx->Nnu; a.nw = ctx->Nw; a.n_iv = ctx->sp.n_iv; a.n_iw = ctx->sp.n_iw; a.shift = ctx->sp.shift;
    a.fft_lo = ctx->fft_lo; a.numax = numax; a.w_per_chunk = wpc;
    a.w_begin = ctx->w_lo; a.w_end = ctx->w_hi;
    a.U = ctx->mp.U; a.lam_m = lam_m; a.lam_d = lam_d; a.part = part;
    a.lam_m_dev = lm_dev; a.lam_d_dev = ld_dev;
    const size_t sm = (size_t)wpc * per;
    auto kern = tc ? k_eom_forward<DIM, M, true> : k_eom_forward<DIM, M, false>;
    LDGA_CUDA(ctx, set_smem(ctx, kern, sm));
    dim3 grid(nchunk, numax);
    StageTimer st_(ctx, LDGA_STAGE_EOM_FORWARD);
    kern<<<grid, tc ? kThr<M, true> : kThr<M, false>, sm, ctx->stream>>>(make_T<M>(ctx), a, ctx->d_ghat, ctx->d_chi[0], ctx->d_gam[0],
                                               ctx->d_chi[1], ctx->d_gam[1], ctx->d_lambda0, ctx->d_partial);
    LDGA_LAUNCHED(ctx, "k_eom_forward");
    nchunk_out = nchunk;
    return LDGA_OK;
}

template <int DIM, int M>
int run_eom_inverse(ldga_ctx* ctx, int numax, int nchunk, const double* d_tail, int tc, double chiloc_m_sum,
                    double2* out, int out_ld, int add_hartree) {
    const bool ttc = ctx->transform_tc;
    const int np = pairs_per_cta<DIM, M>(numax, ttc ? kSmemBudgetTC : kSmemBudget);
    const size_t sm = smem_bytes<DIM, M>(np);
    auto kern = ttc ? k_eom_inverse<DIM, M, true> : k_eom_inverse<DIM, M, false>;
    LDGA_CUDA(ctx, set_smem(ctx, kern, sm));
    dim3 grid((numax + np - 1) / np);
    const double scale = 1.0 / ((double)ctx->Nk * (double)ctx->Nk);
    const double hartree = ctx->mp.n * ctx->mp.U / 2.0;
    if (!ctx->shard_constants) {   // another rank of the ω shards adds the tail and Hartree terms
        tc = 0;
        add_hartree = 0;
    }
    StageTimer st_(ctx, LDGA_STAGE_EOM_INVERSE);
    kern<<<grid, ttc ? kThr<M, true> : kThr<M, false>, sm, ctx->stream>>>(make_T<M>(ctx), numax, nchunk, scale, ctx->mp.beta, ctx->mp.U,
                                               hartree, d_tail, tc, chiloc_m_sum, ctx->d_partial, out, out_ld,
                                               add_hartree, np);
    LDGA_LAUNCHED(ctx, "k_eom_inverse");
    return LDGA_OK;
}

template <int DIM, int M>
int run_gloc_vjp(ldga_ctx* ctx, const double2* chi0_bar, const double2* sbar, int numax, double lam_m, double lam_d,
                 double2* shat, double2* rows, const int32_t* start, const int32_t* idx, double2* gbar_hat,
                 double2* gbar) {
    const int nbub = chi0_bar ? ctx->Nnu * ctx->Nw : 0;
    if (chi0_bar) {
        const int np = pairs_per_cta<DIM, M>(nbub);
        const size_t sm = smem_bytes<DIM, M>(np);
        auto kern = k_bubble_vjp<DIM, M>;
        LDGA_CUDA(ctx, set_smem(ctx, kern, sm));
        dim3 grid((nbub + np - 1) / np);
        const double sb = -ctx->mp.beta / ((double)ctx->Nk * (double)ctx->Nk);
        kern<<<grid, kThreads, sm, ctx->stream>>>(make_T<M>(ctx), ctx->Nnu, ctx->Nw, ctx->sp.n_iv, ctx->sp.n_iw,
                                                   ctx->sp.shift, ctx->fft_lo, sb, ctx->d_kmult, ctx->d_ghat, chi0_bar,
                                                   rows, np);
        LDGA_LAUNCHED(ctx, "k_bubble_vjp");
    }
    if (sbar) {
        {
            const int np = pairs_per_cta<DIM, M>(numax);
            const size_t sm = smem_bytes<DIM, M>(np);
            auto kern = k_vjp_transform<DIM, M>;
            LDGA_CUDA(ctx, set_smem(ctx, kern, sm));
            dim3 grid((numax + np - 1) / np);
            kern<<<grid, kThreads, sm, ctx->stream>>>(make_T<M>(ctx), numax, 0, ctx->d_kmult, sbar, shat, np);
            LDGA_LAUNCHED(ctx, "k_vjp_transform");
        }
        const int total = numax * ctx->Nw;
        const int np = pairs_per_cta<DIM, M>(total);
        const size_t sm = smem_bytes<DIM, M>(np);
        auto kern = k_eom_gvjp<DIM, M>;
        LDGA_CUDA(ctx, set_smem(ctx, kern, sm));
        EomArgs a;
        a.nnu = ctx->Nnu; a.nw = ctx->Nw; a.n_iv = ctx->sp.n_iv; a.n_iw = ctx->sp.n_iw; a.shift = ctx->sp.shift;
        a.fft_lo = ctx->fft_lo; a.numax = numax; a.w_per_chunk = 1;
        a.U = ctx->mp.U; a.lam_m = lam_m; a.lam_d = lam_d; a.part = -1;
        a.lam_m_dev = nullptr; a.lam_d_dev = nullptr;
        dim3 grid((total + np - 1) / np);
        const double c = 1.0 / (ctx->mp.beta * (double)ctx->Nk * (double)ctx->Nk);
        kern<<<grid, kThreads, sm, ctx->stream>>>(make_T<M>(ctx), a, c, ctx->d_kmult, shat, ctx->d_chi[0], ctx->d_gam[0],
                                                   ctx->d_chi[1], ctx->d_gam[1], ctx->d_lambda0,
                                                   rows + (size_t)2 * nbub * ctx->Nq, np);
        LDGA_LAUNCHED(ctx, "k_eom_gvjp");
    }
    k_ghat_gather<<<2 * 148, 256, 0, ctx->stream>>>(ctx->Nf, ctx->Nq, start, idx, rows, gbar_hat);
    LDGA_LAUNCHED(ctx, "k_ghat_gather");
    {
        const int np = pairs_per_cta<DIM, M>(ctx->Nf);
        const size_t sm = smem_bytes<DIM, M>(np);
        auto kern = k_vjp_transform<DIM, M>;
        LDGA_CUDA(ctx, set_smem(ctx, kern, sm));
        dim3 grid((ctx->Nf + np - 1) / np);
        kern<<<grid, kThreads, sm, ctx->stream>>>(make_T<M>(ctx), ctx->Nf, 1, ctx->d_kmult, gbar_hat, gbar, np);
        LDGA_LAUNCHED(ctx, "k_vjp_transform");
    }
    return LDGA_OK;
}

template <int DIM, int M>
int run_eom_vjp(ldga_ctx* ctx, int numax, double lam_m, double lam_d, int tc, const double2* sbar,
                double2* gm_bar, double2* gd_bar, double2* l0_bar, double* xm_bar, double* xd_bar, double2* shat,
                double* cm, double* cd) {
    {   // Ŝbar = S(Sbar / kMult)
        const int np = pairs_per_cta<DIM, M>(numax);
        const size_t sm = smem_bytes<DIM, M>(np);
        auto kern = k_vjp_sbar<DIM, M>;
        LDGA_CUDA(ctx, set_smem(ctx, kern, sm));
        dim3 grid((numax + np - 1) / np);
        kern<<<grid, kThreads, sm, ctx->stream>>>(make_T<M>(ctx), numax, ctx->d_kmult, sbar, shat, np);
        LDGA_LAUNCHED(ctx, "k_vjp_sbar");
    }
    {
        const int total = numax * ctx->Nw;
        const int np = pairs_per_cta<DIM, M>(total);
        const size_t sm = smem_bytes<DIM, M>(np);
        auto kern = k_eom_vjp<DIM, M>;
        LDGA_CUDA(ctx, set_smem(ctx, kern, sm));
        EomVjpArgs a;
        a.nnu = ctx->Nnu; a.nw = ctx->Nw; a.n_iv = ctx->sp.n_iv; a.n_iw = ctx->sp.n_iw; a.shift = ctx->sp.shift;
        a.fft_lo = ctx->fft_lo; a.numax = numax; a.U = ctx->mp.U; a.lam_m = lam_m; a.lam_d = lam_d;
        a.scale = 1.0 / (ctx->mp.beta * (double)ctx->Nk * (double)ctx->Nk);
        dim3 grid((total + np - 1) / np);
        kern<<<grid, kThreads, sm, ctx->stream>>>(make_T<M>(ctx), a, ctx->d_kmult, ctx->d_ghat, shat, ctx->d_chi[0],
                                                   ctx->d_gam[0], ctx->d_chi[1], ctx->d_gam[1], gm_bar, gd_bar, l0_bar,
                                                   cm, cd, np);
        LDGA_LAUNCHED(ctx, "k_eom_vjp");
    }
    if (tc) {
        k_vjp_tail<<<1, 256, 0, ctx->stream>>>(ctx->Nq, numax, ctx->mp.beta, ctx->mp.U, sbar, ctx->d_red + 60);
        LDGA_LAUNCHED(ctx, "k_vjp_tail");
    }
    const double tail_w = tc ? 1.0 / (ctx->mp.beta * (double)ctx->Nk) : 0.0;
    k_eom_vjp_chi<<<2 * 148, 256, 0, ctx->stream>>>(ctx->Nq, ctx->Nw, numax, lam_m, lam_d, tail_w, ctx->d_kmult,
                                                    ctx->d_red + 60, ctx->d_chi[0], ctx->d_chi[1], cm, cd, xm_bar,
                                                    xd_bar);
    LDGA_LAUNCHED(ctx, "k_eom_vjp_chi");
    return LDGA_OK;
}

}  // namespace

#define LDGA_CASE(D, MM)                                  \
    if (ctx->dim == D && ctx->M == MM) { return BODY(D, MM); }

int launch_gloc_transform(ldga_ctx* ctx, bool from_sigma) {
#define BODY(D, MM) run_gloc<D, MM>(ctx, from_sigma)
    LDGA_FOR_EACH_GRID(LDGA_CASE)
#undef BODY
    return ctx_fail(ctx, LDGA_ERR_ARG, "unsupported k-grid size");
}

int launch_bubble(ldga_ctx* ctx) {
    ++ctx->chi0_gen;
#define BODY(D, MM) run_bubble<D, MM>(ctx)
    LDGA_FOR_EACH_GRID(LDGA_CASE)
#undef BODY
    return ctx_fail(ctx, LDGA_ERR_ARG, "unsupported k-grid size");
}

// EoM: forward kernel then inverse kernel; `part` selects the contribution (-1: full EoM; 0..5 the
// calc_Σ_parts pieces).  d_tail: device scalar sum_kω(chi_m^lam) (read only when tc != 0).
namespace {
template <int DIM, int M>
int run_eom_all(ldga_ctx* ctx, int numax, double lam_m, double lam_d, const double* lm_dev, const double* ld_dev,
                int part, const double* d_tail, int tc, double chiloc_m_sum, double2* out, int out_ld,
                int add_hartree) {
    int nchunk = 0;
    int st = run_eom<DIM, M>(ctx, numax, lam_m, lam_d, lm_dev, ld_dev, part, nchunk);
    if (st != LDGA_OK) return st;
    return run_eom_inverse<DIM, M>(ctx, numax, nchunk, d_tail, tc, chiloc_m_sum, out, out_ld, add_hartree);
}
}  // namespace

int launch_eom(ldga_ctx* ctx, int numax, double lam_m, double lam_d, const double* lam_m_dev,
               const double* lam_d_dev, int part, const double* d_tail, int tc, double chiloc_m_sum,
               double2* out, int out_ld, int add_hartree) {
#define BODY(D, MM)                                                                                      \
    run_eom_all<D, MM>(ctx, numax, lam_m, lam_d, lam_m_dev, lam_d_dev, part, d_tail, tc, chiloc_m_sum, out, \
                       out_ld, add_hartree)
    LDGA_FOR_EACH_GRID(LDGA_CASE)
#undef BODY
    return ctx_fail(ctx, LDGA_ERR_ARG, "unsupported k-grid size");
}

int launch_eom_vjp(ldga_ctx* ctx, int numax, double lam_m, double lam_d, int tc, const double2* sbar,
                   double2* gm_bar, double2* gd_bar, double2* l0_bar, double* xm_bar, double* xd_bar, double2* shat,
                   double* cm, double* cd) {
#define BODY(D, MM) run_eom_vjp<D, MM>(ctx, numax, lam_m, lam_d, tc, sbar, gm_bar, gd_bar, l0_bar, xm_bar, xd_bar, shat, cm, cd)
    LDGA_FOR_EACH_GRID(LDGA_CASE)
#undef BODY
    return ctx_fail(ctx, LDGA_ERR_ARG, "unsupported k-grid size");
}

int launch_gloc_vjp(ldga_ctx* ctx, const double2* chi0_bar, const double2* sbar, int numax, double lam_m,
                    double lam_d, double2* shat, double2* rows, const int32_t* start, const int32_t* idx,
                    double2* gbar_hat, double2* gbar) {
#define BODY(D, MM) run_gloc_vjp<D, MM>(ctx, chi0_bar, sbar, numax, lam_m, lam_d, shat, rows, start, idx, gbar_hat, gbar)
    LDGA_FOR_EACH_GRID(LDGA_CASE)
#undef BODY
    return ctx_fail(ctx, LDGA_ERR_ARG, "unsupported k-grid size");
}

int launch_sigma_loc_grad(ldga_ctx* ctx, const double2* gbar, int n_sigma, double2* out) {
    k_sigma_loc_grad<<<n_sigma, 256, 0, ctx->stream>>>(ctx->Nq, ctx->Nf, ctx->fft_lo, n_sigma, ctx->d_gloc, gbar, out);
    LDGA_LAUNCHED(ctx, "k_sigma_loc_grad");
    return LDGA_OK;
}
