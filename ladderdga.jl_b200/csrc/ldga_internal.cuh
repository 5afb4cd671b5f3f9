// Internal definitions of libldga_b200: handle layout, complex helpers, k-grid wedge indexing and
// the symmetry-reduced k-space transform shared by the G setup, the bubble and the EoM kernels.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/ldga_b200.h"

#define LDGA_MAX_M 33        // wedge points per axis: N/2 + 1 for N <= 64
#define LDGA_MAX_NNU 128     // fermionic box size handled by the BSE kernels

// ------------------------------------------------------------------------------------------
// complex helpers (interleaved double2 / float2)
// ------------------------------------------------------------------------------------------
__host__ __device__ __forceinline__ double2 cmk(double r, double i) { return make_double2(r, i); }
__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
// 1/z computed as conj(z)/|z|^2 with a scaling step so that |z|^2 cannot overflow.
__host__ __device__ __forceinline__ double2 cinv(double2 z) {
    double s = fabs(z.x) > fabs(z.y) ? fabs(z.x) : fabs(z.y);
    if (s == 0.0) return make_double2(1.0 / 0.0, 0.0);
    double xr = z.x / s, xi = z.y / s;
    double d = (xr * xr + xi * xi) * s;
    return make_double2(xr / d, -xi / d);
}
__host__ __device__ __forceinline__ double2 cdiv(double2 a, double2 b) { return cmul(a, cinv(b)); }

__host__ __device__ __forceinline__ float2 fadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 fmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// ------------------------------------------------------------------------------------------
// wedge indexing: irreducible points (a >= b [>= c] >= 0), lexicographic order
// ------------------------------------------------------------------------------------------
__host__ __device__ __forceinline__ int widx2(int a, int b) { return a * (a + 1) / 2 + b; }
__host__ __device__ __forceinline__ int widx3(int a, int b, int c) {
    return a * (a + 1) * (a + 2) / 6 + b * (b + 1) / 2 + c;
}
__host__ __device__ __forceinline__ int sidx2(int a, int b) { return a >= b ? widx2(a, b) : widx2(b, a); }
__host__ __device__ __forceinline__ int sidx3(int a, int b, int c) {
    int x = a, y = b, z = c, t;
    if (x < y) { t = x; x = y; y = t; }
    if (y < z) { t = y; y = z; z = t; }
    if (x < y) { t = x; x = y; y = t; }
    return widx3(x, y, z);
}
__host__ __device__ __forceinline__ int wedge_count(int dim, int M) {
    return dim == 2 ? M * (M + 1) / 2 : M * (M + 1) * (M + 2) / 6;
}

// ------------------------------------------------------------------------------------------
// transform matrix, passed by value so that the coefficients sit in the kernel-parameter
// constant bank and feed the FMAs directly:  T[q][m] = w_m cos(2 pi m q / N), w = 1 at m = 0 and
// m = N/2, 2 otherwise.  For a function even in every axis (every array of this library is
// point-group symmetric) the full-grid DFT along one axis equals this cosine sum over m <= N/2.
// ------------------------------------------------------------------------------------------
template <int M>
struct TMat {
    double t[M * M];
};

// ------------------------------------------------------------------------------------------
// handle
// ------------------------------------------------------------------------------------------
struct ldga_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    ldga_lattice lat{};
    ldga_model mp{};
    ldga_sim sp{};
    int prec = LDGA_PREC_FP64;

    int dim = 0, ns = 0, M = 0, Nk = 0, Nq = 0, Nnu = 0, Nw = 0, Nf = 0, fft_lo = 0;
    std::vector<double> kmult, eps, Tmat;   // Tmat: M*M row-major T[q][m]
    std::vector<int32_t> wedge;

    // device arrays (column-major reference layouts, first index fastest)
    double* d_kmult = nullptr;     // [Nq]
    double* d_eps = nullptr;       // [Nq]
    double2* d_ghat = nullptr;     // [Nq, Nf]   transformed G, R on the wedge
    double2* d_gloc = nullptr;     // [Nq, Nf]   G(k, nu)
    double2* d_sigma_loc = nullptr;
    int n_sigma_loc = 0;
    double2* d_chi0 = nullptr;     // [Nq, Nnu, Nw]
    double2* d_Gamma[2] = {nullptr, nullptr};   // [Nnu, Nnu, Nw]
    double* d_chi[2] = {nullptr, nullptr};      // [Nq, Nw]
    double2* d_gam[2] = {nullptr, nullptr};     // [Nq, Nnu, Nw]
    double2* d_F = nullptr;        // [Nnu, Nnu, Nw]
    double2* d_lambda0 = nullptr;  // [Nq, Nnu, Nw]
    double2* d_sigma = nullptr;    // [Nq, numax]
    int sigma_numax = 0;
    double2* d_gladder = nullptr;  // [Nq, Nf]
    double2* d_partial = nullptr;  // EoM partial sums [nchunk, Nq, numax]
    size_t partial_elems = 0;
    double* d_red = nullptr;       // reduction scratch
    int32_t* d_flags = nullptr;    // BSE fallback flags [Nq*Nw]
    int32_t* d_flags2 = nullptr;   // the d channel's flags when both channels run in one launch
    int32_t* d_list = nullptr;     // compacted fallback list (the m channel's list of a pair launch)
    int32_t* d_list2 = nullptr;    // the d channel's list of a pair launch
    double2* d_gamma_t = nullptr;  // MIXED BSE adjoint: Gamma(w) transposed [Nnu, Nnu, Nw]
    int32_t* d_count = nullptr;
    double2* d_pivot_scratch = nullptr;   // pivoted fallback matrices in HBM when N (N+1) does not fit shared memory
    int2* d_bub_pairs = nullptr;          // bubble pairs computed directly (pair, conjugate partner or -1)
    int32_t* d_qperm = nullptr;           // [Nw][Nq] q order of the preconditioned BSE (k_bse_qorder)
    uint64_t chi0_gen = 0;                // bumped whenever chi0 is (re)written on the stream
    uint64_t qperm_gen = ~0ull;           // chi0_gen the q order was computed from (both channels share it)
    unsigned long long* d_iter_stats = nullptr;   // [2] preconditioned BSE: residual passes, warps
    // scratch arena of the adjoint entry points: bump-allocated within a call, reused by later
    // calls; a call that needs more takes extra cudaMalloc blocks and the arena grows to the
    // recorded demand at the start of the next call
    char* d_arena = nullptr;
    size_t arena_cap = 0, arena_used = 0, arena_want = 0;
    int n_bub_pairs = 0;
    // ω shard (ldga_set_omega_shard): the bubble, BSE, lambda_0 and EoM stages cover the bosonic
    // indices [w_lo, w_hi) only; the EoM's 1/iν tail and Hartree terms are added where
    // shard_constants is set (one rank), so the ranks' Σ_ladder add up to the whole one
    int w_lo = 0, w_hi = 0;
    bool shard_constants = true;
    std::vector<int> bub_pair_w_start;    // [Nw + 1] first bubble pair of each ω (pairs are ω-major)

    cudaStream_t own_stream = nullptr;   // created by the handle; `stream` may be a caller's stream
    // ldga_chain_m's copies that overlap its kernels: the vertices and local inputs go in on io_stream
    // while G and the bubble run, chi_m/chi_d come out there while the λ and EoM stages run
    cudaStream_t io_stream = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_gamma = nullptr, ev_loc = nullptr, ev_chi = nullptr, ev_join = nullptr;
    cudaEvent_t ev_bub = nullptr, ev_l0 = nullptr;   // χ₀ ready for λ₀ on io_stream; λ₀ ready for the EoM
    bool l0_beside = true;               // the chain's λ₀ on io_stream (false: in line, for batched chains)
    // λdm residual lanes 1 and 2 (lane 0 is the handle's own stream and buffers): a stream, the
    // EoM's partial sums and Σ of each, and one event per lane marking its μ fit
    bool dm_lanes = true;                // false (LDGA_DM_LANES=0 at ldga_create): residuals one by one
    cudaStream_t dm_stream[2] = {nullptr, nullptr};
    cudaEvent_t dm_ev[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t dm_fork = nullptr;
    double2* dm_partial[2] = {nullptr, nullptr};
    size_t dm_partial_elems[2] = {0, 0};
    double2* dm_sigma[2] = {nullptr, nullptr};
    bool capturing = false;              // a CUDA graph of the chain is being captured

    // fused chain (ldga_chain_m): persistent input buffers and the captured graph
    double2* d_chiloc = nullptr;   // [Nnu, Nnu, Nw] local chi_m
    double2* d_gimp = nullptr;
    int n_gimp_alloc = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    std::vector<uint64_t> graph_key;
    std::vector<std::pair<int, int>> graph_ev;   // stage events recorded inside the captured graph
    int64_t graph_launches = 0;                  // kernels per replay of the captured graph
    double* h_stage = nullptr;     // pinned host staging for the chain's scalars (64 doubles + 4 ints)

    // k-space transforms of the G setup, bubble and EoM on the FP64 tensor path (mma.sync m8n8k4,
    // environment LDGA_TRANSFORM=tc at ldga_create); the CUDA-core form is the default
    bool transform_tc = false;
    // the λm Newton's cluster all-reduce by st.async + mbarrier instead of a cluster barrier per
    // iteration (environment LDGA_NEWTON=barrier at ldga_create selects the barrier form)
    bool newton_async = true;
    // CTAs of the λm Newton's cluster: 16 where the device can place a non-portable 16-CTA cluster
    // (chosen by newton_cluster_size at ldga_create; LDGA_NEWTON_CLUSTER=8 keeps 8), else 8
    int newton_cluster = 8;
    // residual sweeps of MIXED's preconditioned BSE iteration before a matrix is handed to the pivoted
    // FP64 solve (environment LDGA_ITER_SWEEPS at ldga_create, 0..1000; 0 hands every matrix over)
    int iter_sweeps = 40;

    // stage timing (ldga_profile / ldga_stage_times)
    bool profiling = false;
    uint32_t prof_mask = 0;       // stages whose events are recorded while profiling (bit = stage)
    struct EvPair { cudaEvent_t a = nullptr, b = nullptr; };
    std::vector<EvPair> ev_pool;
    std::vector<int> ev_free;
    std::vector<std::pair<int, int>> ev_pending;   // (stage, slot)
    double stage_ms[LDGA_N_STAGES] = {0};
    int stage_cnt[LDGA_N_STAGES] = {0};
    int64_t n_launches = 0;        // kernels launched by this handle

    bool have_ghat = false, have_chi0 = false, have_F = false, have_lambda0 = false, have_sigma = false;
    bool have_Gamma[2] = {false, false}, have_chi[2] = {false, false}, have_gam[2] = {false, false};
    int lambda_dm_evals = 0;

    std::string err;
};

// error helpers (host)
int ctx_fail(ldga_ctx* ctx, int code, const std::string& msg);
int ctx_cuda(ldga_ctx* ctx, cudaError_t e, const char* what);
#define LDGA_CUDA(ctx, call)                                        \
    do {                                                            \
        cudaError_t _e = (call);                                    \
        if (_e != cudaSuccess) return ctx_cuda((ctx), _e, #call);   \
    } while (0)
#define LDGA_LAUNCHED(ctx, what)                                    \
    do {                                                            \
        (ctx)->n_launches++;                                        \
        cudaError_t _e = cudaGetLastError();                        \
        if (_e != cudaSuccess) return ctx_cuda((ctx), _e, what);    \
    } while (0)

// Dynamic shared-memory opt-in for a kernel; skipped while a CUDA graph is being captured (the
// uncaptured warm-up run of the same sequence has already set it).
template <typename F>
inline cudaError_t set_smem(ldga_ctx* c, F* f, size_t sm) {
    if (c->capturing) return cudaSuccess;
    return cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
}

// ω shard helpers: the number of bosonic indices the stages cover, and whether a shard is set
inline int shard_nw(const ldga_ctx* c) { return c->w_hi - c->w_lo; }
inline bool sharded(const ldga_ctx* c) { return c->w_lo != 0 || c->w_hi != c->Nw; }
// entry points whose stages need every ω (the λdm and self-consistent loops, the fused chain, the
// adjoints) refuse a sharded handle
int require_unsharded(ldga_ctx* ctx, const char* what);

bool bse_has_fast_path(int nnu);
// BSE kernel configurations (autotuning): count and name per (Nν, precision), the chosen index,
// and one uncompacted launch of configuration i on the channel's current inputs.
int bse_variant_count(int nnu, int prec);
const char* bse_variant_name(int nnu, int prec, int i);
int bse_tuned_variant(int nnu, int prec);
void bse_set_variant(int nnu, int prec, int i);
void bse_reset_variants();
int bse_run_variant(ldga_ctx* ctx, int channel, int i);
// shared memory of one pivoted-fallback matrix [N][N+1] (complex FP64) plus its reduction scratch
size_t bse_pivot_smem(int nnu);
constexpr size_t LDGA_PIVOT_SMEM_MAX = 220 * 1024;
constexpr int LDGA_PIVOT_GRID = 2 * 148;

// Records CUDA events around one stage when the handle is profiling (no-op otherwise).
struct StageTimer {
    ldga_ctx* c;
    int stage;
    int slot;
    StageTimer(ldga_ctx* ctx, int st);
    ~StageTimer();
};

// kernel launchers implemented in the .cu files
int launch_gloc_transform(ldga_ctx* ctx, bool from_sigma);
int launch_bubble(ldga_ctx* ctx);
// BSE for one channel; enqueues the fallback for flagged matrices on the device (no host sync).
// d_fail (device int32) receives the number of matrices that stayed unsolved.
int launch_bse(ldga_ctx* ctx, int channel, int32_t* d_fail);
int launch_bse_pair(ldga_ctx* ctx, int32_t* d_fail);
// Adjoint of one BSE channel: chi0_bar (written, or added to when accumulate), y and z buffers
// [Nq, Nnu, Nw], Gamma_bar [Nnu, Nnu, Nw]; the number of adjoint solves above the backward-error
// threshold is added to d_fail.
int launch_bse_adj(ldga_ctx* ctx, int channel, const double* chi_bar, const double2* gam_bar, double2* chi0_bar,
                   double2* ybuf, double2* zbuf, double2* gamma_bar, int32_t* d_fail, bool accumulate = false);
// Adjoint of the EoM at (lam_m, lam_d): sbar [numax][Nq] -> gm_bar, gd_bar, l0_bar [Nq, Nnu, Nw] (pre-zeroed;
// any may be null), xm_bar, xd_bar [Nq, Nw] (may be null).  Scratch: shat [numax * Nq] complex,
// cm, cd [numax * Nq * Nw] real.
int launch_eom_vjp(ldga_ctx* ctx, int numax, double lam_m, double lam_d, int tc, const double2* sbar,
                   double2* gm_bar, double2* gd_bar, double2* l0_bar, double* xm_bar, double* xd_bar, double2* shat,
                   double* cm, double* cd);
// Adjoint of the lattice G: bubble part (chi0_bar [Nq, Nnu, Nw], may be null) and the EoM's direct
// use of Ghat (sbar [numax][Nq], may be null) -> rows (scratch, one per term), gathered by the CSR
// lists start/idx per fft_range frequency into gbar_hat [Nf][Nq]; gbar = kMult S(gbar_hat/kMult).
int launch_gloc_vjp(ldga_ctx* ctx, const double2* chi0_bar, const double2* sbar, int numax, double lam_m,
                    double lam_d, double2* shat, double2* rows, const int32_t* start, const int32_t* idx,
                    double2* gbar_hat, double2* gbar);
// Sigma_loc_bar(m), m < n_sigma, from gbar [Nf][Nq] and the handle's G (d_gloc)
int launch_sigma_loc_grad(ldga_ctx* ctx, const double2* gbar, int n_sigma, double2* out);
int launch_F_from_chi(ldga_ctx* ctx, const double2* d_chi_loc, const double2* d_gimp, int n_gimp);
int launch_lambda0(ldga_ctx* ctx);
// chi0_bar += lambda0_bar conj(sum_nu F) / beta^2 (adjoint of launch_lambda0 with F fixed)
int launch_lambda0_vjp(ldga_ctx* ctx, const double2* l0_bar, double2* chi0_bar);
// dE_pot,1/dΣ_ladder [Nq, numax] with μ following the filling condition (calc_E after G_from_Σladder!)
int launch_epot_vjp(ldga_ctx* ctx, int numax, double mu, const double2* sigma, double2* out);
// EoM forward + inverse.  lam_*_dev (may be null) are device scalars added to lam_m / lam_d.
int launch_eom(ldga_ctx* ctx, int numax, double lam_m, double lam_d, const double* lam_m_dev,
               const double* lam_d_dev, int part, const double* d_tail, int tc, double chiloc_m_sum,
               double2* out, int out_ld, int add_hartree);
int launch_sum_kw(ldga_ctx* ctx, int channel, double lam, int mode, double* d_out, const double* lam_dev = nullptr);
int launch_lambda_min(ldga_ctx* ctx, int channel, double* d_out);
// sum_kω(χ_m^λm) and sum_kω(χ_d^λd) (mode 0 of launch_sum_kw) in one launch
int launch_sum_kw2(ldga_ctx* ctx, double lam_m, double lam_d, double* d_out_m, double* d_out_d);
int newton_cluster_size(bool async);
int launch_chi_tail_shift(ldga_ctx* ctx, int channel, double dc2);
// newton_right's defaults (LambdaCorrection/helpers.jl:133): nsteps 100, atol 1e-13.  sum_d_out given:
// rhs = rhs_const - sum_kω(chi_d) is formed in the kernel and the sum stored there (rhs_sub_dev unused);
// sum_m_out given: sum_kω(chi_m) at the final λ is stored there.
int launch_lambda_m(ldga_ctx* ctx, double rhs_const, const double* rhs_sub_dev, double* d_out /*[5]*/,
                    int nsteps = 100, double atol = 1e-13, double* sum_d_out = nullptr,
                    double* sum_m_out = nullptr);
// mu_dev (may be null): device scalar the μ fit starts from instead of mu_in
int launch_g_ladder(ldga_ctx* ctx, int numax, int fix_n, double mu_in, double* d_out /*[4]*/,
                    const double* mu_dev = nullptr);
int launch_g_ladder_full(ldga_ctx* ctx, int numax, const double* mu_dev);
int launch_calc_E(ldga_ctx* ctx, const double2* G, int ldg, const double2* sigma, int numax, double mu,
                  double* d_out);
int launch_fill_tail(ldga_ctx* ctx, int numax, double tnum, double2* out, int out_ld);
double host_G_shell_sum(int N, double beta);
