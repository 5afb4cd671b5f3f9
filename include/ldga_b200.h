/*
 * ldga_b200.h -- C ABI of the B200 (sm_100a) lDGA ladder library (libldga_b200.so).
 *
 * One handle (ldga_ctx) holds one k-grid / frequency box / parameter point and owns all device
 * memory of the ladder chain: bubble -> Bethe-Salpeter (m, d) -> lambda_0 -> equation of motion
 * -> lambda correction.  Every entry point replaces one function of LadderDGA.jl v0.15.1; the
 * citation beside each declaration names the reference interface (file:line, paths inside the
 * LadderDGA.jl repository).
 *
 * Conventions
 *   - Complex arrays are interleaved (re, im) doubles: Julia ComplexF64, C double _Complex.
 *   - Multi-dimensional arrays are column-major with the first index fastest, exactly the memory
 *     layout of the Julia arrays the reference passes around (chi0.data[q, nu, w], Gamma[nu, nu', w],
 *     chi.data[q, w], gamma.data[q, nu, w], Sigma_ladder[q, nu]).
 *   - Array pointers may point to host or to device memory (CUDA unified addressing).  An output
 *     pointer may be NULL: the result then stays on the device, inside the handle, and later calls
 *     use it (pass NULL for the matching input).
 *   - Every function returns LDGA_OK (0) or an error code; ldga_last_error() gives the message.
 *     Calls are synchronous (the stream is synchronised before return) and a handle must not be
 *     used from two threads at once, like the reference's kG caches.
 *   - q runs over the point-group-irreducible wedge q_x >= q_y (>= q_z) >= 0, q_i <= N/2, in
 *     lexicographic order (q = 0 first); ldga_kgrid() returns the wedge, kMult and eps_k.
 */
#ifndef LDGA_B200_H
#define LDGA_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ldga_ctx ldga_ctx;

/* status codes */
#define LDGA_OK          0
#define LDGA_ERR_ARG     1   /* bad argument / shape: the reference's ArgumentError */
#define LDGA_ERR_CUDA    2   /* CUDA runtime error or missing device */
#define LDGA_ERR_STATE   3   /* prerequisite missing, or lambda applied twice (ErrorException) */
#define LDGA_ERR_NUMERIC 4   /* non-finite data or a BSE matrix that could not be solved */
#define LDGA_ERR_NOCONV  5   /* root finding failed (the reference returns NaN / converged=false) */
#define LDGA_ERR_TYPE    6   /* channel not in {m, d}: error("Unkown type") */

/* BSE precision modes (per handle) */
#define LDGA_PREC_FP64_INV 0 /* full FP64 inverse of every (q, w) matrix: the reference's inv! */
#define LDGA_PREC_FP64     1 /* FP64 elimination of the single right-hand side that chi/gamma use */
#define LDGA_PREC_MIXED    2 /* FP32 work refined against FP64 residuals to backward error 1e-14:
                                 a q-shared FP32 preconditioner with FP64 Richardson sweeps, or an
                                 FP32 elimination with FP64 refinement, or the FP64 elimination where
                                 that is fastest (per box size, autotuned) */

#define LDGA_CH_M 0
#define LDGA_CH_D 1

/* Lattice: simple cubic, eps_k = -2t sum_i cos k_i (2D adds -4t' cos kx cos ky - 2t''(cos 2kx + cos 2ky)).
 * Replaces Dispersions.gen_kGrid("<dim>Dsc-t[-tp-tpp]", ns) (called at runHelpers.jl:88); ns = 1 is
 * the one-point grid of the local quantities (gen_kGrid(kind, 1), runHelpers.jl:134). */
typedef struct {
    int32_t dim;            /* 2 or 3 */
    int32_t ns;             /* points per axis */
    double t, tp, tpp;
} ldga_lattice;

/* ModelParameters (Config.jl:39-47) */
typedef struct {
    double U, mu, beta, n, sVk, Epot_DMFT, Ekin_DMFT;
} ldga_model;

/* SimulationParameters (Config.jl:66-75); chi_helper must be `nothing` (plain path) */
typedef struct {
    int32_t n_iw, n_iv, n_iv_shell, shift;
    int32_t fft_lo, fft_hi;               /* fft_range = fft_lo:fft_hi */
    double usable_prct_reduction;
    int32_t dbg_full_eom_omega;
} ldga_sim;

/* ---------------------------------------------------------------- handle ---------------- */

/* Allocate a handle on CUDA device `device` (gen_kGrid, runHelpers.jl:88, plus the model and
 * simulation parameter structs).  precision is one of LDGA_PREC_*. */
int ldga_create(const ldga_lattice* lat, const ldga_model* mp, const ldga_sim* sp,
                int32_t precision, int32_t device, ldga_ctx** out);
int ldga_destroy(ldga_ctx* ctx);
const char* ldga_last_error(const ldga_ctx* ctx);
const char* ldga_status_string(int32_t status);
int ldga_version(void);

/* Run the handle's work on the caller's CUDA stream (a cudaStream_t; NULL: the handle's own
 * stream).  No reference counterpart: lets a host application order the ladder kernels with its own. */
int ldga_set_stream(ldga_ctx* ctx, void* stream);

/* Per-stage device timing with CUDA events on the handle's stream (no reference counterpart; the
 * reference times stages with TimerOutputs, DepsInit.jl:71).  enable != 0 starts accumulating;
 * ldga_stage_times returns, per stage, total milliseconds and launch counts (LDGA_N_STAGES each). */
#define LDGA_N_STAGES 10
#define LDGA_STAGE_GLOC 0
#define LDGA_STAGE_BUBBLE 1
#define LDGA_STAGE_BSE 2
#define LDGA_STAGE_BSE_FALLBACK 3
#define LDGA_STAGE_LAMBDA0 4
#define LDGA_STAGE_SUMS 5
#define LDGA_STAGE_LAMBDA_NEWTON 6
#define LDGA_STAGE_EOM_FORWARD 7
#define LDGA_STAGE_EOM_INVERSE 8
#define LDGA_STAGE_GLADDER 9
int ldga_profile(ldga_ctx* ctx, int32_t enable);
/* Profile only the stages whose bits are set in mask (bit LDGA_STAGE_*; 0 turns profiling off).  Every
 * stage's events are nodes of the chain's CUDA graph and delay it: timing one stage needs only its own. */
int ldga_profile_stages(ldga_ctx* ctx, uint32_t mask);
int ldga_stage_times(ldga_ctx* ctx, double* ms, int32_t* counts);
/* Number of kernels this handle has launched since it was created. */
int ldga_launch_count(const ldga_ctx* ctx, int64_t* n);

/* Replace the model parameters (e.g. a new mu); mutable ModelParameters, Config.jl:39. */
int ldga_set_model(ldga_ctx* ctx, const ldga_model* mp);
/* ω shard of one parameter point over several handles (one per GPU): the reference's partition of
 * the bosonic frequencies over workers (gen_ω_part / par_partition, parallelization_helpers.jl:22-53;
 * calc_bubble_par / calc_χγ_par / calc_Σ_par, ladderDGATools.jl:46-245).  After the call,
 * ldga_bubble, ldga_bse, ldga_lambda0 and ldga_eom cover the indices [w_lo, w_hi) of 0..Nw-1 only
 * (arrays keep the whole layout; entries outside the shard are not written).  ldga_eom then returns
 * this shard's part of Sigma_ladder; the 1/(i nu) tail and the Hartree term are added only where
 * constants != 0, so the shards' parts sum to the whole Sigma_ladder (given the whole chi_m).
 * The sums, lambda_min and the lambda_m Newton read the whole chi arrays (set them with
 * ldga_set_chi after gathering the shards).  ldga_chain_m, ldga_batch_chain_m, ldga_lambda_dm,
 * ldga_run_sc, ldga_eom_parts and the adjoints return LDGA_ERR_STATE on a sharded handle.
 * ldga_set_omega_shard(ctx, 0, Nw, 1) restores the whole range. */
int ldga_set_omega_shard(ldga_ctx* ctx, int32_t w_lo, int32_t w_hi, int32_t constants);
int ldga_set_precision(ldga_ctx* ctx, int32_t precision);

/* k-grid of the handle: kG.kMult, kG.ϵkGrid and the wedge coordinates (Dispersions.jl; used at
 * DataTypes.jl:230-241 and GFTools.jl:117-126).  Any output may be NULL. */
int ldga_kgrid(const ldga_ctx* ctx, int32_t* nk, int32_t* nq, double* kmult, double* eps,
               int32_t* wedge /* [nq * dim] */);

/* ---------------------------------------------------------------- a1: G and its transforms -- */

/* Lattice G(k, nu) = 1/(i nu_n + mu - eps_k - Sigma_loc(nu_n)) for nu_n in fft_range, and its
 * k-space transform, kept on the device (setup loop runHelpers.jl:113-130, G_fft helpers.jl:153-183).
 * sigma_loc: Sigma_loc(n) for n = 0..n_sigma-1 (n_sigma > max|fft_range|); negative n by
 * conjugation.  gloc_out (may be NULL): gLoc[q, nu] [Nq, Nf]. */
int ldga_gloc(ldga_ctx* ctx, const double* sigma_loc, int32_t n_sigma, double* gloc_out);

/* Use a given G[q, nu] ([Nq, Nf], nu over fft_range) instead, e.g. a ladder G for the
 * self-consistent loop (G_rfft!, helpers.jl:164-173). */
int ldga_set_gloc(ldga_ctx* ctx, const double* gloc);

/* ---------------------------------------------------------------- a2: bubble ----------------- */

/* chi0[q, nu, w] = -beta/N_k sum_k G(k, nu) G(k+q, nu+w) (calc_bubble, BSETools.jl:157-172).
 * chi0_out: [Nq, Nnu, Nw] complex or NULL. */
int ldga_bubble(ldga_ctx* ctx, double* chi0_out);

/* Upload an external chi0 [Nq, Nnu, Nw] (calc_chi_gamma(type, Gamma, chi0, ...) with a user chi0). */
int ldga_set_chi0(ldga_ctx* ctx, const double* chi0);

/* ---------------------------------------------------------------- a7: Bethe-Salpeter --------- */

/* Per (q, w): A = Gamma_r(w) + diag(1/chi0(q, :, w)); chi_r(q,w) = Re(1^T A^-1 1)/beta^2;
 * gamma_r(q, nu, w) = (1^T A^-1)_nu / (chi0(q,nu,w) (1 + s U chi_r)), s = -1 (d), +1 (m)
 * (calc_χγ, BSETools.jl:192-248, inv! LapackWrapper.jl:64-72).
 * gamma_r_in: Gamma_r [Nnu, Nnu, Nw] complex (NULL: reuse the last one of this channel).
 * chi_out [Nq, Nw] real, gam_out [Nq, Nnu, Nw] complex, either may be NULL.
 * n_fallback (may be NULL): matrices re-solved by the pivoted FP64 path. */
int ldga_bse(ldga_ctx* ctx, int32_t channel, const double* gamma_r_in, double* chi_out,
             double* gam_out, int32_t* n_fallback);

/* Vector-Jacobian product of ldga_bse for one channel (the adjoint the reference differentiates
 * through zgetri in inv!, LapackWrapper.jl:64-72, for calc_χγ, BSETools.jl:192-248): given upstream
 * gradients of a real loss with respect to that channel's last chi_r [Nq, Nw] (real) and
 * gamma_r [Nq, Nnu, Nw] (complex, dL/dRe + i dL/dIm), either may be NULL for zero, returns
 *   Gamma_bar [Nnu, Nnu, Nw] = dL/dGamma_r   and   chi0_bar [Nq, Nnu, Nw] = dL/dchi0
 * in the same convention (either output may be NULL).  One FP64 adjoint solve per (q, w) with the
 * untransposed vertex, verified by its backward error; n_flagged (may be NULL) counts solves
 * above 1e-12.  The forward solution is rebuilt from gamma_r and chi_r, not recomputed. */
int ldga_bse_vjp(ldga_ctx* ctx, int32_t channel, const double* chi_bar, const double* gam_bar,
                 double* Gamma_bar, double* chi0_bar, int32_t* n_flagged);

/* Vector-Jacobian product of ldga_eom (calc_Σ, ladderDGATools_singleCore.jl:49-136) at (lam_m,
 * lam_d, numax, tc) on the handle's current chi, gamma, lambda_0 and G transform: given the
 * upstream gradient of a real loss with respect to Sigma_ladder [Nq, numax] (complex, dL/dRe +
 * i dL/dIm), returns dL/d chi_m, dL/d chi_d [Nq, Nw] (real; through the λ correction and the tail
 * term's sum_kω) and dL/d gamma_m, dL/d gamma_d, dL/d lambda_0 [Nq, Nnu, Nw] (complex; zero at the
 * ν the EoM does not read).  Any output may be NULL.  Each (ν_n, ω) term is one transform-product-
 * transform pass, the adjoint of the forward's convolution. */
int ldga_eom_vjp(ldga_ctx* ctx, double lam_m, double lam_d, int32_t numax, int32_t tc, const double* sigma_bar,
                 double* chi_m_bar, double* gam_m_bar, double* chi_d_bar, double* gam_d_bar, double* lambda0_bar);

/* Vector-Jacobian product of the lattice G (the setup loop runHelpers.jl:113-130 with the bubble,
 * BSETools.jl:157-172, and the EoM's G(k, ν+ω), ladderDGATools_singleCore.jl:49-81) for a real loss:
 *   chi0_bar [Nq, Nnu, Nw] = dL/dchi0 (e.g. from ldga_bse_vjp of both channels),
 *   lambda0_bar [Nq, Nnu, Nw] = dL/dlambda_0 (through lambda_0 = chi0 sum_nu F / beta^2, F fixed),
 *   sigma_bar [Nq, numax] = dL/dSigma_ladder with the EoM at (lam_m, lam_d) -- its direct use of G,
 * any of them may be NULL, all complex (dL/dRe + i dL/dIm) ->
 *   sigma_loc_bar [n_sigma] = dL/dSigma_loc(nu_n), n = 0..n_sigma-1 (negative nu by conjugation), and
 *   gloc_bar [Nq, Nf] = dL/dG(q, nu) on the wedge over fft_range (either output may be NULL).
 * mu, G_imp, F_m and the local vertices are held fixed. */
int ldga_gloc_vjp(ldga_ctx* ctx, const double* chi0_bar, const double* lambda0_bar, const double* sigma_bar,
                  double lam_m, double lam_d, int32_t numax, int32_t n_sigma, double* sigma_loc_bar, double* gloc_bar);

/* The whole ladder chain's vector-Jacobian product at fixed λ in one call, every intermediate on
 * the device: ldga_eom_vjp, then ldga_bse_vjp of both channels (their chi0_bar summed), the
 * λ_0 term and ldga_gloc_vjp -- what a ChainRulesCore rrule of calc_bubble → calc_χγ(:m, :d) →
 * calc_λ0 → calc_Σ (BSETools.jl:157-248, ladderDGATools_singleCore.jl:49-136) would pull back.
 * Input sigma_bar [Nq, numax] = dL/dSigma_ladder (complex) for the EoM at (lam_m, lam_d, tc) on the
 * handle's current chi, gamma, lambda_0 (e.g. right after ldga_chain_m).  Outputs (any may be NULL):
 * Gamma_m_bar, Gamma_d_bar [Nnu, Nnu, Nw], sigma_loc_bar [n_sigma] = dL/dSigma_loc(nu_n) through the
 * lattice G, chi0_bar [Nq, Nnu, Nw] = the total dL/dchi0.  Pointers may be host or device memory.
 * n_flagged (may be NULL): adjoint solves of both channels above the backward-error threshold. */
int ldga_chain_vjp(ldga_ctx* ctx, const double* sigma_bar, double lam_m, double lam_d, int32_t numax, int32_t tc,
                   double* Gamma_m_bar, double* Gamma_d_bar, int32_t n_sigma, double* sigma_loc_bar,
                   double* chi0_bar, int32_t* n_flagged);

/* Gradient of E_pot,1 (calc_E, thermodynamics.jl:142-168, on G_from_Σladder!, GFTools.jl:154-186)
 * with respect to Sigma_ladder [Nq, numax] (complex, dE/dRe + i dE/dIm), μ following the filling
 * condition the μ fit solves (μ = the fitted value).  The piece of the λdm implicit derivative
 * that goes through the energies. */
int ldga_epot_vjp(ldga_ctx* ctx, int32_t numax, double mu, const double* sigma, double* sigma_bar);

/* Tile-shape autotuning of the BSE kernel (no reference counterpart; the reference has one LAPACK
 * path).  Every fast-path box size has a few compiled configurations per precision mode (threads
 * per matrix, CTAs per SM the register allocation allows); this times each one `reps` times on the
 * channel's current chi0 and Gamma_r, records the fastest for (Nnu, precision mode) in the process,
 * and leaves that channel's chi and gamma as ldga_bse would.  variant / ms (may be NULL): the chosen
 * index (0 = the default) and its time per launch (-1 when there was only one configuration).
 * Later launches -- including graphs captured afterwards -- use the choice. */
int ldga_autotune_bse(ldga_ctx* ctx, int32_t channel, int32_t reps, int32_t* variant, double* ms);
/* Save / load the recorded choices as text lines "bse <Nnu> <precision> <configuration name>";
 * unknown names are ignored on load. */
int ldga_tune_save(const char* path);
int ldga_tune_load(const char* path);
/* Name of BSE configuration `index` for (nnu, precision) -- index < 0: the one in use -- or NULL. */
const char* ldga_bse_config_name(int32_t nnu, int32_t precision, int32_t index);
/* Work counters of the MIXED preconditioned BSE since the last call (no reference counterpart:
 * diagnostics for rooflines): passes = residual evaluations summed over warps (each warp iterates
 * its q in lockstep), warps = warps that ran.  Both are reset by the call. */
int ldga_bse_sweeps(ldga_ctx* ctx, int64_t* passes, int64_t* warps);
/* Forget every recorded choice: all box sizes use their default configuration again. */
int ldga_tune_reset(void);
/* Device self-test of the tensor-core group inverse that the MIXED BSE's preconditioner uses (no
 * reference counterpart; it stands in for LapackWrapper.jl's inverse inside the preconditioner):
 * Newton-Schulz iterations X <- X (2I - b X) on tcgen05 tensor cores (TF32 operands, FP32
 * accumulation in tensor memory), one CTA on the current device.  b, x0, x_out: n x n complex,
 * row-major interleaved FP32 host arrays (n = 40).  its >= 0: x_out = the iterate after `its`
 * iterations from x0, err_out[0] = max_i sum_j |I - b X|_ij of the iterate before the last update;
 * its < 0: x_out = the single product b x0 (TF32 factors), err_out[0] = 0.  Returns LDGA_ERR_ARG
 * for other n, LDGA_ERR_NUMERIC when a tensor-core completion wait ran out. */
int ldga_selftest_group_inverse(int32_t n, const float* b, const float* x0, int32_t its, float* x_out,
                                float* err_out);

/* Copy a device-resident array of the handle to `out` (host or device) without recomputing it.
 * No reference counterpart: the reference's arrays live in Julia memory; here they stay in HBM
 * until asked for.  what: one of LDGA_GET_*; channel only for chi and gamma. */
#define LDGA_GET_CHI0 0      /* [Nq, Nnu, Nw] complex */
#define LDGA_GET_CHI 1       /* [Nq, Nw] real */
#define LDGA_GET_GAMMA 2     /* [Nq, Nnu, Nw] complex */
#define LDGA_GET_LAMBDA0 3   /* [Nq, Nnu, Nw] complex */
#define LDGA_GET_SIGMA 4     /* [Nq, numax] complex, numax of the last EoM */
#define LDGA_GET_GLOC 5      /* [Nq, Nf] complex */
int ldga_get(ldga_ctx* ctx, int32_t what, int32_t channel, double* out);

/* Upload chi_r [Nq, Nw] / gamma_r [Nq, Nnu, Nw] produced elsewhere (the chiT/gammaT data). */
int ldga_set_chi(ldga_ctx* ctx, int32_t channel, const double* chi);
int ldga_set_gamma(ldga_ctx* ctx, int32_t channel, const double* gam);

/* ---------------------------------------------------------------- a5/a6: F and lambda_0 ------ */

/* F_m(nu, nu', w) from the local chi_m(nu, nu', w) and G_imp (F_from_χ, BSETools.jl:40-53).
 * gimp: G_imp(n) for n = 0..n_gimp-1 (negative n by conjugation).  F_out [Nnu, Nnu, Nw] or NULL. */
int ldga_F_from_chi(ldga_ctx* ctx, const double* chi_loc, const double* gimp, int32_t n_gimp,
                    double* F_out);

/* lambda0[q, nu', w] = chi0[q, nu', w]/beta^2 * sum_nu F[nu, nu', w] (calc_λ0 plain branch,
 * BSETools.jl:129-141).  F_in NULL: the F of the last ldga_F_from_chi.  lambda0_out or NULL. */
int ldga_lambda0(ldga_ctx* ctx, const double* F_in, double* lambda0_out);
int ldga_set_lambda0(ldga_ctx* ctx, const double* lambda0);

/* lambda_0 without any device allocation (no counterpart in the reference; it exists for callers
 * that cannot allocate device memory: a host application whose device memory is entirely owned by
 * its own pool allocator, or code that enqueues work while a stream capture forbids cudaMalloc).
 * Same arithmetic as ldga_lambda0; no handle is needed.  chi0 [nq, nnu, nw], F [nnu, nnu, nw] and
 * lambda0_out [nq, nnu, nw] must be device pointers on the current device; work is enqueued on
 * `stream` (NULL: the legacy default stream) and the call returns without synchronising.
 * Scratch: a built-in device array of 32768 (nu', w) columns (512 KiB, held by every GPU that loads
 * the library until exit); nnu*nw above that is rejected with LDGA_ERR_ARG.  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress), so make that first call before
 * any stream capture.  The address is kept for the life of the process: after cudaDeviceReset on a
 * device, do not call this entry point on that device again.  Pointers into another GPU's memory
 * are rejected with LDGA_ERR_ARG.  Calls share the array: calls that overlap on one GPU race. */
int ldga_lambda0_noalloc(const double* chi0, const double* F, int32_t nq, int32_t nnu, int32_t nw,
                         double beta, double* lambda0_out, void* stream);

/* ---------------------------------------------------------------- a8/a11: sums --------------- */

/* sum_kω with the c2/w^2 tail (DataTypes.jl:215-249) of chi_r transformed by chi_lambda(., lam)
 * (deriv = 0) or by its derivative dchi_lambda (deriv = 1) (LambdaCorrection/helpers.jl:18,61). */
int ldga_sum_kw(ldga_ctx* ctx, int32_t channel, double lam, int32_t deriv, double* out);

/* sum_ωk (DataTypes.jl:257-264): the same sum with the w sum taken first for every q, then the
 * k integration (the reference's consistency check of sum_kω). */
int ldga_sum_wk(ldga_ctx* ctx, int32_t channel, double lam, double* out);

/* get_λ_min (LambdaCorrection/helpers.jl:217-220) of chi_r. */
int ldga_lambda_min(ldga_ctx* ctx, int32_t channel, double* out);

/* ---------------------------------------------------------------- a9/a10: EoM ---------------- */

/* Sigma_ladder[q, nu_n], nu_n = 0..numax-1 (calc_Σ, ladderDGATools_singleCore.jl:108-136 with
 * calc_Σ! :71-81, eom ladderDGATools.jl:260, conv_tmp_add! ladderDGATools.jl:147-160):
 * Sigma = (1/beta) sum_w conv(K_{nu w}, G_{nu+w}) - U (sum_kω chi_m^lam - chiloc_m_sum)/(i nu_n)
 *         + U n/2, K = eom(U, gamma_m, gamma_d, chi_m^lam_m, chi_d^lam_d, lambda0).
 * tc = 0 drops the tail term.  sigma_out [Nq, numax] complex or NULL. */
int ldga_eom(ldga_ctx* ctx, double lam_m, double lam_d, int32_t numax, int32_t tc,
             double chiloc_m_sum, double* sigma_out);

/* calc_Σ_parts (ladderDGATools_singleCore.jl:153-189): [Nq, n_iv, 7] complex, contributions
 * chi_m, gamma_m, chi_d, gamma_d, -U, lambda0 + Hartree, tail. */
int ldga_eom_parts(ldga_ctx* ctx, double lam_m, double lam_d, int32_t tc, double chiloc_m_sum,
                   double* parts_out);

/* ---------------------------------------------------------------- a12/a13: lambda_m ---------- */

/* newton_right (LambdaCorrection/helpers.jl:133-153, nsteps 100, atol 1e-13) on
 * f(l) = sum_kω chi_λ(chi_m, l) - rhs, start 0, bound get_λ_min (λm_correction,
 * conditions_new.jl:144-154), all on the device.  iterations may be NULL. */
int ldga_lambda_m(ldga_ctx* ctx, double rhs, double* lam_out, int32_t* iterations);

/* ldga_lambda_m with newton_right's keywords (helpers.jl:133: nsteps >= 1, atol >= 0).  Once the
 * iteration state (x0, xi) repeats (near the root |f| can stay above atol while xi cycles among a
 * few values ulps apart), whole periods up to nsteps are skipped; lam_out and iterations are bit
 * for bit those of the full loop.  period [2] (may be NULL) receives the iteration at which the
 * repeat was recognised and its period, {0, 0} if nothing was skipped. */
int ldga_lambda_m_newton(ldga_ctx* ctx, double rhs, int32_t nsteps, double atol, double* lam_out,
                         int32_t* iterations, int32_t* period);

/* ---------------------------------------------------------------- a15: G_ladder, energies ---- */

/* From the Sigma_ladder of the last ldga_eom: fit mu to the filling n (fix_n != 0; G_from_Σladder!,
 * GFTools.jl:162-186, filling_pos :255-273), build G_ladder over fft_range, and compute
 * (E_kin, E_pot) (calc_E, thermodynamics.jl:142-168) and the filling n.
 * sigma_loc (n = 0..n_sigma-1, NULL: the last one given to ldga_gloc) fills nu beyond numax.
 * G_out [Nq, Nf] complex or NULL. */
int ldga_g_ladder(ldga_ctx* ctx, const double* sigma_loc, int32_t n_sigma, int32_t fix_n,
                  double mu_in, double* mu_out, double* G_out, double* e_kin, double* e_pot,
                  double* n_out);

/* Upload a Sigma_ladder [Nq, numax] (nu_n = 0..numax-1) as the handle's current self-energy, e.g. a
 * user-modified one before ldga_g_ladder (G_from_Σladder takes Sigma as an argument, GFTools.jl:154). */
int ldga_set_sigma(ldga_ctx* ctx, const double* sigma, int32_t numax);

/* calc_E(G, Σ, μ, kG, mP) (thermodynamics.jl:142-168) for given G, Sigma [Nq, numax] over
 * nu_n = 0..numax-1 (NULL: the handle's G_ladder / Sigma_ladder). */
int ldga_calc_E(ldga_ctx* ctx, const double* G, const double* sigma, int32_t numax, double mu,
                double* e_kin, double* e_pot);

/* ---------------------------------------------------------------- fused chain ---------------- */

/* The plain lambda_m chain of scripts/run_minimal.jl:7-14 for one parameter point, as one call:
 * ldga_gloc -> ldga_bubble -> ldga_bse(m) -> ldga_bse(d) -> ldga_F_from_chi -> ldga_lambda0 ->
 * λm_correction_full (conditions_new.jl:174-190: rhs = 2 imp_density - sum_kω chi_d, device Newton,
 * EoM at numax = Nnu/2, μ fit, energies).  Everything is enqueued without host round trips; with
 * use_graph != 0 and pinned-host or device pointers the sequence is captured once in a CUDA graph
 * and replayed while the pointers and scalars stay the same.
 * Inputs (host or device): sigma_loc [n_sigma], gamma_m, gamma_d, chi_loc_m [Nnu, Nnu, Nw], gimp [n_gimp].
 * Outputs (may be NULL): sigma_out [Nq, Nnu/2], chi_m_out, chi_d_out [Nq, Nw], scalars_out[8] =
 * {λm, μ, E_kin, E_pot1, E_pot2, PP_p2, Newton iterations, filling}. */
int ldga_chain_m(ldga_ctx* ctx, const double* sigma_loc, int32_t n_sigma, const double* gamma_m,
                 const double* gamma_d, const double* chi_loc_m, const double* gimp, int32_t n_gimp,
                 double imp_density, double chiloc_m_sum, int32_t use_graph, double* sigma_out,
                 double* chi_m_out, double* chi_d_out, double* scalars_out);

/* Arguments of ldga_chain_m for one parameter point of a batch. */
typedef struct ldga_chain_io {
    const double* sigma_loc;
    int32_t n_sigma;
    const double* gamma_m;
    const double* gamma_d;
    const double* chi_loc_m;
    const double* gimp;
    int32_t n_gimp;
    double imp_density;
    double chiloc_m_sum;
    double* sigma_out;     /* may be NULL */
    double* chi_m_out;     /* may be NULL */
    double* chi_d_out;     /* may be NULL */
    double* scalars_out;   /* [8] as ldga_chain_m, may be NULL */
} ldga_chain_io;

/* The lambda_m chain for n parameter points, one handle each (any mix of k-grids, frequency boxes
 * and devices): an uneven (U, β) scan in one call.  The reference runs such scans as separate
 * jobs (one run_minimal.jl per point); its per-point path is what ldga_chain_m replaces.  Every
 * point's chain (its captured graph after the first call) is enqueued on its handle's stream
 * before the first host wait, so points of different Nν overlap on the GPU.
 * status[i] (may be NULL) receives each point's status; the return value is the first non-zero
 * one (ldga_last_error of that handle has the message). */
int ldga_batch_chain_m(int32_t n, ldga_ctx* const* ctxs, const ldga_chain_io* io, int32_t use_graph,
                       int32_t* status);

/* ---------------------------------------------------------------- a14: lambda_dm ------------- */

/* λdm_correction plain branch (conditions_new.jl:219-324): 2-D newton_right with a forward-
 * difference Jacobian (helpers.jl:165-208) on
 *   F(lm, ld) = [ (sum chi_d^ld + sum chi_m^lm)/2 - n/2(1-n/2),  E_pot,1 - E_pot,2 ],
 * each evaluation = EoM + mu fit + energies on the device.  numax <= 0: min(n_iv, floor(3 Nw/8)).
 * out7 (may be NULL): [n, mu, E_kin, E_pot1, E_pot2, PP_p1, PP_p2] at the root; numax_out the
 * EoM frequency count used; sigma_out [Nq, numax] and G_out [Nq, Nf] (may be NULL): Sigma_ladder
 * and G_ladder at the root.
 * Returns LDGA_ERR_NOCONV (with lam = NaN) when the root search fails, like the reference's
 * [NaN, NaN]; *converged is the reference's validation flag. */
int ldga_lambda_dm(ldga_ctx* ctx, double chiloc_m_sum, int32_t numax, double lam_min_delta,
                   double atol, int32_t nsteps, double* lam_m, double* lam_d, int32_t* converged,
                   double* out7, int32_t* numax_out, double* sigma_out, double* G_out);

/* run_sc / run_sc! (conditions_new.jl:342-556): the self-consistent ladder loop.  Each iteration:
 * EoM at (lam_m, lam_d) on the current G transform -> linear mixing of Sigma_ladder with the previous
 * one (from the second iteration) -> G_from_Σladder! (μ fit when fit_mu) -> calc_E -> the transform of
 * G_ladder feeds the next EoM; it stops when E_pot,1 and E_pot,2 change by less than conv_abs, or after
 * maxit iterations.  flags:
 *   LDGA_SC_REDO_DM (types :dm, :pre_dm): from the second iteration λ is found again by
 *     λdm_correction on the current G, starting from the previous root; otherwise (types :fix, :m,
 *     :pre_m) λ stays fixed -- the reference's `type == [:pre_m, :m]` test is never true, so :m keeps
 *     its first λ as well;
 *   LDGA_SC_UPDATE_CHI_TAIL (update_χ_tail = true, :519-545): after the loop both channels' c2 tail
 *     is set to E_kin (update_tail!, which shifts chi by Re(Δc2/(i w)^2)), the sum rules are evaluated
 *     again and, unless they hold to conv_abs or 20 updates were made, the loop restarts at it = 1;
 *     the handle's chi and tail coefficient (ldga_model.Ekin_DMFT) are restored on return;
 *   LDGA_SC_LAMBDA_TYPE (types :m, :dm, :pre_m, :pre_dm): a restarted loop takes its first λ from
 *     χ.λ, which is 0 after the first pass (run_sc! resets χ in its first iteration).
 * A flags value of 0 or 1 keeps the meaning of the former redo_dm argument.
 * numax <= 0: min(n_iv, floor(3 Nw / 8)).  The handle's G and its transform are restored on return
 * (the reference iterates on a deepcopy of gLoc_rfft).
 * out[12] = {λm, λd, rhs_c1, lhs_c1, E_pot_1, E_pot_2, E_kin, n, μ, sc_converged, iterations, νmax};
 * sigma_out [Nq, νmax] and G_out [Nq, Nf] (the last Sigma_ladder / G_ladder) may be NULL. */
#define LDGA_SC_REDO_DM 1
#define LDGA_SC_UPDATE_CHI_TAIL 2
#define LDGA_SC_LAMBDA_TYPE 4
int ldga_run_sc(ldga_ctx* ctx, double lam_m, double lam_d, int32_t flags, double mu, double chiloc_m_sum,
                int32_t numax, int32_t maxit, double mixing, double conv_abs, int32_t fit_mu, double lam_min_delta,
                double* out, double* sigma_out, double* G_out);

/* Number of residual evaluations of the last ldga_lambda_dm. */
int ldga_lambda_dm_evals(const ldga_ctx* ctx, int32_t* n_evals);

#ifdef __cplusplus
}
#endif

#endif /* LDGA_B200_H */
