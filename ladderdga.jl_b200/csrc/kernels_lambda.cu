// a5/a6 (F, lambda_0), a8/a11-a13 (Matsubara sums, lambda_m Newton) and a15 (mu fit, G_ladder,
// energies).  The root finders run inside one CTA so that no host round trip sits between
// iterations; every reduction has a fixed summation order, so reruns are bitwise identical.
#include <cmath>

#include "ldga_internal.cuh"

namespace {

constexpr int kRedThreads = 1024;

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
// Deterministic block sum; result valid in every thread.  `red` holds >= 33 doubles.
__device__ double block_sum(double v, double* red) {
    v = warp_sum(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    if (w == 0) {
        double r = (l < (int)(blockDim.x >> 5)) ? red[l] : 0.0;
        r = warp_sum(r);
        if (l == 0) red[32] = r;
    }
    __syncthreads();
    return red[32];
}

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

// colF[nu', w] = sum_nu F[nu, nu', w] in order nu = 0..Nnu-1
__global__ void k_colsum_F(int nnu, int nw, const double2* __restrict__ F, double2* __restrict__ colF) {
    const int total = nnu * nw;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        const int vp = e % nnu, w = e / nnu;
        double2 acc = make_double2(0.0, 0.0);
        const double2* col = F + ((size_t)w * nnu + vp) * nnu;
        for (int v = 0; v < nnu; ++v) acc = cadd(acc, col[v]);
        colF[e] = acc;
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

// ---------------------------------------------------------------------------------------------
// sum_kω (DataTypes.jl:230-249):  (sum_w [ sum_q kMult f(chi)/N_k - c2/(i w)^2 ] - beta^2 c2/12)/beta
// f = chi_lambda(., lam) (deriv 0) or dchi_lambda (deriv 1)
// ---------------------------------------------------------------------------------------------
struct SumArgs {
    int nq, nw, n_iw;
    double beta, c2, inv_nk;
};

__device__ __forceinline__ double chi_l(double x, double lam) { return x / (lam * x + 1.0); }

__device__ double sum_kw_block(const SumArgs& a, const double* __restrict__ chi, const double* __restrict__ kmult,
                               double lam, int deriv, double* red) {
    double acc = 0.0;
    const int total = a.nq * a.nw;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
        const int q = e % a.nq;
        double v = chi[e];
        if (deriv) {
            const double t = chi_l(v, lam);
            v = -t * t;
        } else if (lam != 0.0) {
            v = chi_l(v, lam);
        }
        acc = fma(kmult[q], v, acc);
    }
    const double s = block_sum(acc, red) * a.inv_nk;
    // tail: sum over w != 0 of real(c2/(i w_m)^2) = -c2 beta^2/(4 pi^2 m^2)
    double tail = 0.0;
    for (int m = 1; m <= a.n_iw; ++m) tail += 2.0 * (-a.c2 * a.beta * a.beta / (4.0 * M_PI * M_PI * (double)m * m));
    return (s - tail + (-a.beta * a.beta / 12.0) * a.c2) / a.beta;
}

// sum_ωk order: per q, (sum_w [chi - tail] - beta^2 c2/12)/beta, then the kMult-weighted mean
__device__ double sum_wk_block(const SumArgs& a, const double* __restrict__ chi, const double* __restrict__ kmult,
                               double lam, double* red) {
    double tail = 0.0;
    for (int m = 1; m <= a.n_iw; ++m) tail += 2.0 * (-a.c2 * a.beta * a.beta / (4.0 * M_PI * M_PI * (double)m * m));
    double acc = 0.0;
    for (int q = threadIdx.x; q < a.nq; q += blockDim.x) {
        double s = 0.0;
        for (int w = 0; w < a.nw; ++w) {
            const double v = chi[(size_t)w * a.nq + q];
            s += lam != 0.0 ? chi_l(v, lam) : v;
        }
        s = (s - tail + a.c2 * (-a.beta * a.beta / 12.0)) / a.beta;
        acc = fma(kmult[q], s, acc);
    }
    return block_sum(acc, red) * a.inv_nk;
}

__global__ void __launch_bounds__(kRedThreads) k_sum_kw(SumArgs a, const double* chi, const double* kmult,
                                                          double lam, int deriv, double* out) {
    __shared__ double red[40];
    const double r = deriv == 2 ? sum_wk_block(a, chi, kmult, lam, red) : sum_kw_block(a, chi, kmult, lam, deriv, red);
    if (threadIdx.x == 0) out[0] = r;
}

__global__ void __launch_bounds__(kRedThreads) k_lambda_min(int nq, int w0, const double* chi, double* out) {
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
__global__ void __launch_bounds__(kRedThreads) k_lambda_m(SumArgs a, const double* chi, const double* kmult,
                                                            double rhs, double xmin, int nsteps, double atol,
                                                            double* out) {
    __shared__ double red[40];
    const double delta = 1e-4;
    double x0 = 0.0, xi = x0;
    int i = 1;
    while (true) {
        const double fi = sum_kw_block(a, chi, kmult, xi, 0, red) - rhs;
        const double dfi = sum_kw_block(a, chi, kmult, xi, 1, red);
        const double dfii = 1.0 / dfi;
        xi = x0 - dfii * fi;
        if (fabs(fi) < atol) break;
        if (xi < xmin) x0 = xmin + delta + fabs(xmin - x0) / 2.0;
        else x0 = xi;
        if (i >= nsteps) break;
        ++i;
    }
    if (threadIdx.x == 0) { out[0] = xi; out[1] = (double)i; }
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

// f(mu) = filling_pos - n and df/dmu, summed over q (kMult) and nu_n < numax
__device__ void filling_f_df(const GArgs& a, const double* kmult, const double* eps, const double2* sigma,
                             double mu, double* red, double& f, double& df) {
    double sre = 0.0, dre = 0.0;
    const int total = a.nq * a.numax;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
        const int q = e % a.nq, nn = e / a.nq;
        const double2 G = g_at(mu, eps[q], sigma[e], nn, a.beta);
        const double2 G2 = cmul(G, G);
        sre = fma(kmult[q], G.x, sre);
        dre = fma(kmult[q], -G2.x, dre);
    }
    const double sG = block_sum(sre, red) * a.inv_nk;
    const double dG = block_sum(dre, red) * a.inv_nk;
    f = 2.0 * (2.0 * sG / a.beta + 0.5 + mu * a.shell) / (1.0 + a.U * a.shell) - a.n;
    df = 2.0 * (2.0 * dG / a.beta + a.shell) / (1.0 + a.U * a.shell);
}

__global__ void __launch_bounds__(kRedThreads) k_mu_fit_energy(GArgs a, const double* kmult, const double* eps,
                                                                 const double2* sigma, int fix_n, double mu_in,
                                                                 double mu_ref, double* out) {
    __shared__ double red[40];
    double mu = mu_in;
    bool failed = false;
    if (fix_n) {
        // safeguarded Newton (same method as the oracle's mu_newton)
        double lo = -INFINITY, hi = INFINITY;
        const double tol = 1e-14;
        for (int it = 0; it < 100; ++it) {
            double f, df;
            filling_f_df(a, kmult, eps, sigma, mu, red, f, df);
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
    // energies at mu (calc_E with mu_ref = the chemical potential handed to calc_E) and filling
    const double hartree = a.n * a.U / 2.0;
    double ekin = 0.0, epot = 0.0, sre = 0.0;
    const int total = a.nq * a.numax;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
        const int q = e % a.nq, nn = e / a.nq;
        const double2 G = g_at(mu, eps[q], sigma[e], nn, a.beta);
        const double wn = (2.0 * nn + 1.0) * M_PI / a.beta;
        const double tail = -1.0 / (wn * wn);                           // 1/(i w)^2
        const double ekin_tc = eps[q] + hartree - mu;
        const double epot_tc = a.U * a.U * 0.5 * a.n * (1.0 - 0.5 * a.n) + hartree * (eps[q] + hartree - mu);
        const double2 GS = cmul(G, sigma[e]);
        const double ep = GS.x - epot_tc * tail;
        const double ek = eps[q] * (G.x - ekin_tc * tail);
        ekin = fma(kmult[q], 4.0 * ek, ekin);
        epot = fma(kmult[q], 2.0 * ep, epot);
        sre = fma(kmult[q], G.x, sre);
    }
    // tail_inv terms (once per q)
    for (int q = threadIdx.x; q < a.nq; q += blockDim.x) {
        const double ekin_tc = eps[q] + hartree - mu;
        const double epot_tc = a.U * a.U * 0.5 * a.n * (1.0 - 0.5 * a.n) + hartree * (eps[q] + hartree - mu);
        const double epot_inv = (a.beta / 2.0) * hartree + (a.beta / 2.0) * (-a.beta / 2.0) * epot_tc;
        const double ekin_inv = (a.beta / 2.0) * eps[q] * (1.0 + -a.beta * ekin_tc);
        ekin = fma(kmult[q], ekin_inv, ekin);
        epot = fma(kmult[q], epot_inv, epot);
    }
    const double Ek = block_sum(ekin, red) * a.inv_nk / a.beta;
    const double Ep = block_sum(epot, red) * a.inv_nk / a.beta;
    const double sG = block_sum(sre, red) * a.inv_nk;
    const double nfill = 2.0 * (2.0 * sG / a.beta + 0.5 + mu * a.shell) / (1.0 + a.U * a.shell);
    (void)mu_ref;
    if (threadIdx.x == 0) { out[0] = mu; out[1] = Ek; out[2] = Ep; out[3] = nfill; }
}

// calc_E for a given G (column stride ldg) and Sigma over nu_n = 0..numax-1 (thermodynamics.jl:142-168)
__global__ void __launch_bounds__(kRedThreads) k_calc_E(GArgs a, const double* kmult, const double* eps,
                                                          const double2* G, int ldg, const double2* sigma,
                                                          double mu, double* out) {
    __shared__ double red[40];
    const double hartree = a.n * a.U / 2.0;
    double ekin = 0.0, epot = 0.0;
    const int total = a.nq * a.numax;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
        const int q = e % a.nq, nn = e / a.nq;
        const double2 g = G[(size_t)nn * ldg + q];
        const double wn = (2.0 * nn + 1.0) * M_PI / a.beta;
        const double tail = -1.0 / (wn * wn);
        const double ekin_tc = eps[q] + hartree - mu;
        const double epot_tc = a.U * a.U * 0.5 * a.n * (1.0 - 0.5 * a.n) + hartree * (eps[q] + hartree - mu);
        const double2 GS = cmul(g, sigma[e]);
        ekin = fma(kmult[q], 4.0 * (eps[q] * (g.x - ekin_tc * tail)), ekin);
        epot = fma(kmult[q], 2.0 * (GS.x - epot_tc * tail), epot);
    }
    for (int q = threadIdx.x; q < a.nq; q += blockDim.x) {
        const double ekin_tc = eps[q] + hartree - mu;
        const double epot_tc = a.U * a.U * 0.5 * a.n * (1.0 - 0.5 * a.n) + hartree * (eps[q] + hartree - mu);
        ekin = fma(kmult[q], (a.beta / 2.0) * eps[q] * (1.0 + -a.beta * ekin_tc), ekin);
        epot = fma(kmult[q], (a.beta / 2.0) * hartree + (a.beta / 2.0) * (-a.beta / 2.0) * epot_tc, epot);
    }
    const double Ek = block_sum(ekin, red) * a.inv_nk / a.beta;
    const double Ep = block_sum(epot, red) * a.inv_nk / a.beta;
    if (threadIdx.x == 0) { out[0] = Ek; out[1] = Ep; }
}

// G_ladder over fft_range: Sigma_ladder for nu_n < numax, Sigma_loc beyond, negative nu by conjugation
__global__ void k_g_ladder_full(int nq, int nf, int fft_lo, int numax, double beta, double mu,
                                const double* eps, const double2* sigma, const double2* sigma_loc,
                                double2* G) {
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
            // G(-n-1)... G_new[:, first:-1] = conj(G_new[:, last-1:-1:0])
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

SumArgs sum_args(const ldga_ctx* ctx) {
    SumArgs a;
    a.nq = ctx->Nq; a.nw = ctx->Nw; a.n_iw = ctx->sp.n_iw;
    a.beta = ctx->mp.beta; a.c2 = ctx->mp.Ekin_DMFT; a.inv_nk = 1.0 / (double)ctx->Nk;
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
    k_F_from_chi<<<256, 256, 0, ctx->stream>>>(ctx->Nnu, ctx->Nw, ctx->sp.n_iv, ctx->sp.n_iw, ctx->sp.shift,
                                              ctx->mp.beta, d_chi_loc, d_gimp, ctx->d_F);
    LDGA_LAUNCHED(ctx, "k_F_from_chi");
    return LDGA_OK;
}

int launch_lambda0(ldga_ctx* ctx) {
    double2* colF = reinterpret_cast<double2*>(ctx->d_red + 64);
    k_colsum_F<<<64, 256, 0, ctx->stream>>>(ctx->Nnu, ctx->Nw, ctx->d_F, colF);
    LDGA_LAUNCHED(ctx, "k_colsum_F");
    k_lambda0<<<4 * 148, 256, 0, ctx->stream>>>(ctx->Nq, ctx->Nnu, ctx->Nw, 1.0 / (ctx->mp.beta * ctx->mp.beta),
                                                ctx->d_chi0, colF, ctx->d_lambda0);
    LDGA_LAUNCHED(ctx, "k_lambda0");
    return LDGA_OK;
}

int launch_sum_kw(ldga_ctx* ctx, int channel, double lam, int deriv, double* d_out) {
    k_sum_kw<<<1, kRedThreads, 0, ctx->stream>>>(sum_args(ctx), ctx->d_chi[channel], ctx->d_kmult, lam, deriv, d_out);
    LDGA_LAUNCHED(ctx, "k_sum_kw");
    return LDGA_OK;
}

int launch_lambda_min(ldga_ctx* ctx, int channel, double* d_out) {
    const int w0 = (ctx->Nw + 1) / 2 - 1;   // ω0_index = ceil(Nw/2), 1-based
    k_lambda_min<<<1, kRedThreads, 0, ctx->stream>>>(ctx->Nq, w0, ctx->d_chi[channel], d_out);
    LDGA_LAUNCHED(ctx, "k_lambda_min");
    return LDGA_OK;
}

int launch_lambda_m(ldga_ctx* ctx, double rhs, double* d_out) {
    // lambda_min first (device), then the Newton loop reads it back from the host copy
    int st = launch_lambda_min(ctx, LDGA_CH_M, d_out + 2);
    if (st) return st;
    double xmin = 0.0;
    LDGA_CUDA(ctx, cudaMemcpyAsync(&xmin, d_out + 2, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    LDGA_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    k_lambda_m<<<1, kRedThreads, 0, ctx->stream>>>(sum_args(ctx), ctx->d_chi[LDGA_CH_M], ctx->d_kmult, rhs, xmin,
                                                   100, 1e-13, d_out);
    LDGA_LAUNCHED(ctx, "k_lambda_m");
    return LDGA_OK;
}

int launch_g_ladder(ldga_ctx* ctx, int numax, int fix_n, double mu_in, double* d_out) {
    GArgs a;
    a.nq = ctx->Nq; a.numax = numax; a.beta = ctx->mp.beta; a.U = ctx->mp.U; a.n = ctx->mp.n;
    a.inv_nk = 1.0 / (double)ctx->Nk;
    a.shell = host_G_shell_sum(numax + 1, ctx->mp.beta);
    k_mu_fit_energy<<<1, kRedThreads, 0, ctx->stream>>>(a, ctx->d_kmult, ctx->d_eps, ctx->d_sigma, fix_n, mu_in,
                                                        mu_in, d_out);
    LDGA_LAUNCHED(ctx, "k_mu_fit_energy");
    return LDGA_OK;
}

int launch_calc_E(ldga_ctx* ctx, const double2* G, int ldg, const double2* sigma, int numax, double mu,
                  double* d_out) {
    GArgs a;
    a.nq = ctx->Nq; a.numax = numax; a.beta = ctx->mp.beta; a.U = ctx->mp.U; a.n = ctx->mp.n;
    a.inv_nk = 1.0 / (double)ctx->Nk;
    a.shell = 0.0;
    k_calc_E<<<1, kRedThreads, 0, ctx->stream>>>(a, ctx->d_kmult, ctx->d_eps, G, ldg, sigma, mu, d_out);
    LDGA_LAUNCHED(ctx, "k_calc_E");
    return LDGA_OK;
}

int launch_g_ladder_full(ldga_ctx* ctx, int numax, double mu) {
    k_g_ladder_full<<<4 * 148, 256, 0, ctx->stream>>>(ctx->Nq, ctx->Nf, ctx->fft_lo, numax, ctx->mp.beta, mu,
                                                      ctx->d_eps, ctx->d_sigma, ctx->d_sigma_loc, ctx->d_gladder);
    LDGA_LAUNCHED(ctx, "k_g_ladder_full");
    return LDGA_OK;
}

int launch_fill_tail(ldga_ctx* ctx, int numax, double tnum, double2* out, int out_ld) {
    k_fill_tail<<<64, 256, 0, ctx->stream>>>(ctx->Nq, numax, ctx->mp.beta, tnum, out, out_ld);
    LDGA_LAUNCHED(ctx, "k_fill_tail");
    return LDGA_OK;
}
