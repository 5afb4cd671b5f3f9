// C ABI of libldga_b200 (declarations and reference citations in include/ldga_b200.h).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "ldga_internal.cuh"

double host_G_shell_sum(int N, double beta);
int launch_fill_tail(ldga_ctx* ctx, int numax, double tnum, double2* out, int out_ld);
int launch_calc_E(ldga_ctx* ctx, const double2* G, int ldg, const double2* sigma, int numax, double mu,
                  double* d_out);

static thread_local std::string g_create_error;

int ctx_fail(ldga_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->err = msg;
    else g_create_error = msg;
    return code;
}

int ctx_cuda(ldga_ctx* ctx, cudaError_t e, const char* what) {
    return ctx_fail(ctx, LDGA_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

int require_unsharded(ldga_ctx* ctx, const char* what) {
    if (ctx && sharded(ctx))
        return ctx_fail(ctx, LDGA_ERR_STATE, std::string(what) + " needs every bosonic frequency: the handle covers "
                                                 "the ω shard [" + std::to_string(ctx->w_lo) + ", " +
                                                 std::to_string(ctx->w_hi) + "); reset it with ldga_set_omega_shard");
    return LDGA_OK;
}

// While a graph is captured the two event records become graph nodes; their (stage, slot) pairs are
// kept with the graph and read after every replay (ldga_chain_m).
StageTimer::StageTimer(ldga_ctx* ctx, int st) : c(ctx), stage(st), slot(-1) {
    if (!c || !c->profiling || !((c->prof_mask >> st) & 1u)) return;
    if (c->ev_free.empty()) {
        ldga_ctx::EvPair p;
        if (cudaEventCreate(&p.a) != cudaSuccess || cudaEventCreate(&p.b) != cudaSuccess) return;
        c->ev_pool.push_back(p);
        c->ev_free.push_back((int)c->ev_pool.size() - 1);
    }
    slot = c->ev_free.back();
    c->ev_free.pop_back();
    // inside a capture only "external" records become event-record nodes that can be timed later
    cudaEventRecordWithFlags(c->ev_pool[slot].a, c->stream, c->capturing ? cudaEventRecordExternal : 0);
}

StageTimer::~StageTimer() {
    if (slot < 0) return;
    cudaEventRecordWithFlags(c->ev_pool[slot].b, c->stream, c->capturing ? cudaEventRecordExternal : 0);
    if (c->capturing) c->graph_ev.emplace_back(stage, slot);
    else c->ev_pending.emplace_back(stage, slot);
}

namespace {

template <typename T>
int dev_alloc(ldga_ctx* ctx, T** p, size_t n) {
    if (*p) return LDGA_OK;
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(n, 1) * sizeof(T));
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "cudaMalloc");
    return LDGA_OK;
}

// copy between any two pointers (host or device) on the handle's stream
int copy(ldga_ctx* ctx, void* dst, const void* src, size_t bytes) {
    if (bytes == 0) return LDGA_OK;
    LDGA_CUDA(ctx, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, ctx->stream));
    return LDGA_OK;
}

int sync(ldga_ctx* ctx) {
    LDGA_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    LDGA_CUDA(ctx, cudaGetLastError());
    return LDGA_OK;
}

struct DeviceGuard {
    int prev = 0;
    explicit DeviceGuard(int dev) { cudaGetDevice(&prev); if (prev != dev) cudaSetDevice(dev); }
    ~DeviceGuard() { int cur = 0; cudaGetDevice(&cur); if (cur != prev) cudaSetDevice(prev); }
};

#define TRY(x) do { int _s = (x); if (_s != LDGA_OK) return _s; } while (0)
#define NEED(ctx, cond, msg) do { if (!(cond)) return ctx_fail((ctx), LDGA_ERR_STATE, (msg)); } while (0)

// doubles per λdm residual slot (dm_slot); three slots follow the λ₀ scratch at the end of d_red
constexpr int kDmSlot = 10;

bool supported_grid(int dim, int M) {
    static const int m2[] = {1, 2, 3, 4, 5, 6, 7, 9, 11, 13, 17, 21, 25, 33};
    static const int m3[] = {1, 2, 3, 4, 5, 6, 7, 9, 11, 13, 17};
    if (dim == 2) return std::find(std::begin(m2), std::end(m2), M) != std::end(m2);
    if (dim == 3) return std::find(std::begin(m3), std::end(m3), M) != std::end(m3);
    return false;
}

// point-group reduced simple-cubic grid: wedge (a >= b [>= c]), multiplicities, eps_k, T matrix
void build_kgrid(ldga_ctx* c) {
    const int N = c->ns, M = N / 2 + 1, d = c->dim;
    c->M = M;
    c->Nk = d == 2 ? N * N : N * N * N;
    c->Nq = wedge_count(d, M);
    c->kmult.assign(c->Nq, 0.0);
    c->eps.assign(c->Nq, 0.0);
    c->wedge.assign((size_t)c->Nq * d, 0);
    auto fold = [N](int n) { return std::min(n, (N - n) % N); };
    if (d == 2) {
        for (int x = 0; x < N; ++x)
            for (int y = 0; y < N; ++y) c->kmult[sidx2(fold(x), fold(y))] += 1.0;
        for (int a = 0; a < M; ++a)
            for (int b = 0; b <= a; ++b) {
                const int q = widx2(a, b);
                c->wedge[(size_t)q * 2] = a; c->wedge[(size_t)q * 2 + 1] = b;
                const double kx = 2.0 * M_PI * a / N, ky = 2.0 * M_PI * b / N;
                c->eps[q] = -2.0 * c->lat.t * (cos(kx) + cos(ky)) - 4.0 * c->lat.tp * cos(kx) * cos(ky) -
                            2.0 * c->lat.tpp * (cos(2 * kx) + cos(2 * ky));
            }
    } else {
        for (int x = 0; x < N; ++x)
            for (int y = 0; y < N; ++y)
                for (int z = 0; z < N; ++z) c->kmult[sidx3(fold(x), fold(y), fold(z))] += 1.0;
        for (int a = 0; a < M; ++a)
            for (int b = 0; b <= a; ++b)
                for (int cc = 0; cc <= b; ++cc) {
                    const int q = widx3(a, b, cc);
                    c->wedge[(size_t)q * 3] = a; c->wedge[(size_t)q * 3 + 1] = b; c->wedge[(size_t)q * 3 + 2] = cc;
                    c->eps[q] = -2.0 * c->lat.t * (cos(2.0 * M_PI * a / N) + cos(2.0 * M_PI * b / N) +
                                                   cos(2.0 * M_PI * cc / N));
                }
    }
    // T[q][m] = w_m cos(2 pi m q / N); w_m = 1 for m = 0 and m = N/2 (N even), else 2
    c->Tmat.assign((size_t)M * M, 0.0);
    for (int q = 0; q < M; ++q)
        for (int m = 0; m < M; ++m) {
            const double w = (m == 0 || (N % 2 == 0 && 2 * m == N)) ? 1.0 : 2.0;
            // exact integer reduction of the phase keeps the cosines symmetric to the last bit
            const long ph = ((long)m * q) % N;
            c->Tmat[(size_t)q * M + m] = w * cos(2.0 * M_PI * (double)ph / (double)N);
        }
}

int alloc_all(ldga_ctx* c) {
    const size_t nq = c->Nq, nnu = c->Nnu, nw = c->Nw, nf = c->Nf;
    TRY(dev_alloc(c, &c->d_kmult, nq));
    TRY(dev_alloc(c, &c->d_eps, nq));
    TRY(dev_alloc(c, &c->d_ghat, nq * nf));
    TRY(dev_alloc(c, &c->d_gloc, nq * nf));
    TRY(dev_alloc(c, &c->d_chi0, nq * nnu * nw));
    for (int r = 0; r < 2; ++r) {
        TRY(dev_alloc(c, &c->d_Gamma[r], nnu * nnu * nw));
        TRY(dev_alloc(c, &c->d_chi[r], nq * nw));
        TRY(dev_alloc(c, &c->d_gam[r], nq * nnu * nw));
    }
    TRY(dev_alloc(c, &c->d_F, nnu * nnu * nw));
    TRY(dev_alloc(c, &c->d_lambda0, nq * nnu * nw));
    TRY(dev_alloc(c, &c->d_sigma, nq * std::max<size_t>(nnu, 1)));
    TRY(dev_alloc(c, &c->d_gladder, nq * nf));
    TRY(dev_alloc(c, &c->d_red, 64 + 2 * nnu * nw + 64 + 3 * kDmSlot));
    TRY(dev_alloc(c, &c->d_flags, nq * nw));
    TRY(dev_alloc(c, &c->d_list, nq * nw));
    TRY(dev_alloc(c, &c->d_count, 4));
    TRY(dev_alloc(c, &c->d_qperm, nq * nw));
    TRY(dev_alloc(c, &c->d_iter_stats, 2));
    LDGA_CUDA(c, cudaMemset(c->d_iter_stats, 0, 2 * sizeof(unsigned long long)));
    if (bse_pivot_smem((int)nnu) > LDGA_PIVOT_SMEM_MAX)
        TRY(dev_alloc(c, &c->d_pivot_scratch, (size_t)LDGA_PIVOT_GRID * nnu * (nnu + 1)));
    {   // bubble representatives: pair (vi, wi) and its conjugate partner nu'' = -nu - w - 1 in the box
        std::vector<int2> pairs;
        std::vector<char> done(nnu * nw, 0);
        for (int wi = 0; wi < (int)nw; ++wi)
            for (int vi = 0; vi < (int)nnu; ++vi) {
                const int pi = vi + (int)nnu * wi;
                if (done[pi]) continue;
                const int wn = wi - c->sp.n_iw, sh = c->sp.shift * (wn / 2);
                const int vn = (vi - c->sp.n_iv) - sh;
                const int vi2 = (-vn - wn - 1) + c->sp.n_iv + sh;
                int pj = -1;
                if (vi2 >= 0 && vi2 < (int)nnu && vi2 != vi) {
                    pj = vi2 + (int)nnu * wi;
                    done[pj] = 1;
                }
                done[pi] = 1;
                pairs.push_back(make_int2(pi, pj));
            }
        c->n_bub_pairs = (int)pairs.size();
        // the list is ω-major (a pair and its partner share ω): first pair of each ω for shards
        c->bub_pair_w_start.assign(nw + 1, c->n_bub_pairs);
        for (int p = c->n_bub_pairs - 1; p >= 0; --p) c->bub_pair_w_start[pairs[p].x / (int)nnu] = p;
        for (int w = (int)nw - 1; w >= 0; --w)
            c->bub_pair_w_start[w] = std::min(c->bub_pair_w_start[w], c->bub_pair_w_start[w + 1]);
        c->w_lo = 0;
        c->w_hi = (int)nw;
        TRY(dev_alloc(c, &c->d_bub_pairs, pairs.size()));
        TRY(copy(c, c->d_bub_pairs, pairs.data(), pairs.size() * sizeof(int2)));
        TRY(sync(c));   // the host vector goes out of scope
    }
    TRY(copy(c, c->d_kmult, c->kmult.data(), nq * sizeof(double)));
    TRY(copy(c, c->d_eps, c->eps.data(), nq * sizeof(double)));
    return sync(c);
}

void free_all(ldga_ctx* c) {
    void* ptrs[] = {c->d_kmult, c->d_eps, c->d_ghat, c->d_gloc, c->d_sigma_loc, c->d_chi0, c->d_Gamma[0],
                    c->d_Gamma[1], c->d_chi[0], c->d_chi[1], c->d_gam[0], c->d_gam[1], c->d_F, c->d_lambda0,
                    c->d_sigma, c->d_gladder, c->d_partial, c->d_red, c->d_flags, c->d_flags2, c->d_list, c->d_list2, c->d_gamma_t, c->d_count,
                    c->d_pivot_scratch, c->d_bub_pairs, c->d_arena, c->d_qperm, c->d_iter_stats,
                    c->dm_partial[0], c->dm_partial[1], c->dm_sigma[0], c->dm_sigma[1]};
    for (void* p : ptrs)
        if (p) cudaFree(p);
}

// device scratch of one call (e.g. an adjoint), released on every exit path.  Buffers are carved
// from the handle's arena (256-byte aligned); what does not fit is cudaMalloc'ed and freed at the
// end, and the arena is regrown to the call's total demand when the next call opens its scratch
// (every entry point synchronises its stream before returning, so no kernel still uses it).
struct DevScratch {
    ldga_ctx* c = nullptr;
    size_t mark = 0, demand = 0;
    std::vector<void*> own;
    int open(ldga_ctx* ctx) {
        c = ctx;
        mark = ctx->arena_used;
        if (mark == 0 && ctx->arena_want > ctx->arena_cap) {
            if (ctx->d_arena) cudaFree(ctx->d_arena);
            ctx->d_arena = nullptr;
            ctx->arena_cap = 0;
            cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&ctx->d_arena), ctx->arena_want);
            if (e != cudaSuccess) {
                ctx->d_arena = nullptr;
                return ctx_cuda(ctx, e, "cudaMalloc (adjoint scratch)");
            }
            ctx->arena_cap = ctx->arena_want;
        }
        return LDGA_OK;
    }
    template <typename T>
    int get(ldga_ctx* ctx, T** out, size_t n) {
        *out = nullptr;
        if (!c) TRY(open(ctx));
        const size_t bytes = (std::max<size_t>(n, 1) * sizeof(T) + 255) & ~size_t(255);
        demand += bytes;
        ctx->arena_want = std::max(ctx->arena_want, mark + demand);
        if (ctx->arena_used + bytes <= ctx->arena_cap) {
            *out = reinterpret_cast<T*>(ctx->d_arena + ctx->arena_used);
            ctx->arena_used += bytes;
            return LDGA_OK;
        }
        TRY(dev_alloc(ctx, out, n));
        own.push_back(*out);
        return LDGA_OK;
    }
    ~DevScratch() {
        for (void* x : own) cudaFree(x);
        if (c) c->arena_used = mark;
    }
};

// The lattice-G adjoint on device buffers: chi0_bar (bubble, may be null) and sbar [numax][Nq] (the
// EoM's direct use of G, numax = 0: none) -> G_bar [Nf, Nq] (*gb) and, for n_sigma > 0,
// Sigma_loc_bar [n_sigma] (*slb).  The CSR lists of rows per fft_range frequency are built here
// in increasing row order; start and idx must outlive the stream's copies (the caller syncs).
int gloc_vjp_device(ldga_ctx* ctx, DevScratch& sc, const double2* d_c0b, const double2* d_sb, int numax, double lam_m,
                    double lam_d, int n_sigma, std::vector<int32_t>& start, std::vector<int32_t>& idx,
                    double2** slb, double2** gb) {
    const size_t nfq = (size_t)ctx->Nf * ctx->Nq;
    const bool bub = d_c0b != nullptr;
    const int nbub = bub ? ctx->Nnu * ctx->Nw : 0, neom = numax * ctx->Nw;
    std::vector<std::vector<int32_t>> lists(ctx->Nf);
    for (int wi = 0; wi < ctx->Nw && bub; ++wi)
        for (int vi = 0; vi < ctx->Nnu; ++vi) {
            const int pi = vi + ctx->Nnu * wi, wn = wi - ctx->sp.n_iw;
            const int vn = (vi - ctx->sp.n_iv) - ctx->sp.shift * (wn / 2);
            lists[vn - ctx->fft_lo].push_back(2 * pi);
            lists[vn + wn - ctx->fft_lo].push_back(2 * pi + 1);
        }
    for (int wi = 0; wi < ctx->Nw && numax > 0; ++wi)
        for (int n = 0; n < numax; ++n) {
            const int wn = wi - ctx->sp.n_iw;
            lists[n + wn - ctx->fft_lo].push_back(2 * nbub + n + numax * wi);
        }
    for (auto& l : lists) std::sort(l.begin(), l.end());
    start.assign(ctx->Nf + 1, 0);
    idx.clear();
    for (int f = 0; f < ctx->Nf; ++f) {
        start[f + 1] = start[f] + (int)lists[f].size();
        idx.insert(idx.end(), lists[f].begin(), lists[f].end());
    }
    double2 *d_shat = nullptr, *d_rows = nullptr, *d_ghb = nullptr;
    int32_t *d_start = nullptr, *d_idx = nullptr;
    if (numax > 0) TRY(sc.get(ctx, &d_shat, (size_t)ctx->Nq * numax));
    TRY(sc.get(ctx, &d_rows, (size_t)(2 * nbub + neom + 1) * ctx->Nq));
    TRY(sc.get(ctx, &d_start, start.size()));
    TRY(sc.get(ctx, &d_idx, std::max<size_t>(idx.size(), 1)));
    TRY(copy(ctx, d_start, start.data(), start.size() * sizeof(int32_t)));
    if (!idx.empty()) TRY(copy(ctx, d_idx, idx.data(), idx.size() * sizeof(int32_t)));
    TRY(sc.get(ctx, &d_ghb, nfq));
    TRY(sc.get(ctx, gb, nfq));
    TRY(launch_gloc_vjp(ctx, d_c0b, numax > 0 ? d_sb : nullptr, numax, lam_m, lam_d, d_shat, d_rows, d_start, d_idx,
                        d_ghb, *gb));
    if (n_sigma > 0) {
        TRY(sc.get(ctx, slb, (size_t)n_sigma));
        TRY(launch_sigma_loc_grad(ctx, *gb, n_sigma, *slb));
    }
    return LDGA_OK;
}

int set_sigma_loc(ldga_ctx* ctx, const double* sigma_loc, int n_sigma) {
    const int L = std::max(std::abs(ctx->sp.fft_lo), std::abs(ctx->sp.fft_hi));
    if (n_sigma <= L)
        return ctx_fail(ctx, LDGA_ERR_ARG, "Sigma_loc must cover n = 0..max|fft_range| (" + std::to_string(L + 1) +
                                               " values), got " + std::to_string(n_sigma));
    if (n_sigma > ctx->n_sigma_loc) {
        if (ctx->d_sigma_loc) cudaFree(ctx->d_sigma_loc);
        ctx->d_sigma_loc = nullptr;
        TRY(dev_alloc(ctx, &ctx->d_sigma_loc, (size_t)n_sigma));
    }
    ctx->n_sigma_loc = n_sigma;
    return copy(ctx, ctx->d_sigma_loc, sigma_loc, (size_t)n_sigma * sizeof(double2));
}

}  // namespace

// =============================================================================================
extern "C" {

int ldga_version(void) { return 1; }

const char* ldga_status_string(int32_t s) {
    switch (s) {
        case LDGA_OK: return "ok";
        case LDGA_ERR_ARG: return "invalid argument";
        case LDGA_ERR_CUDA: return "CUDA error";
        case LDGA_ERR_STATE: return "invalid state";
        case LDGA_ERR_NUMERIC: return "numerical failure";
        case LDGA_ERR_NOCONV: return "root finding did not converge";
        case LDGA_ERR_TYPE: return "unknown channel type";
        default: return "unknown status";
    }
}

const char* ldga_last_error(const ldga_ctx* ctx) { return ctx ? ctx->err.c_str() : g_create_error.c_str(); }

int ldga_create(const ldga_lattice* lat, const ldga_model* mp, const ldga_sim* sp, int32_t precision,
                int32_t device, ldga_ctx** out) {
    if (!lat || !mp || !sp || !out) return ctx_fail(nullptr, LDGA_ERR_ARG, "null argument");
    *out = nullptr;
    if (lat->dim != 2 && lat->dim != 3) return ctx_fail(nullptr, LDGA_ERR_ARG, "lattice dimension must be 2 or 3");
    if (lat->ns < 1 || lat->ns > 64) return ctx_fail(nullptr, LDGA_ERR_ARG, "points per axis must be 1..64");
    if (sp->n_iv < 1 || sp->n_iw < 0) return ctx_fail(nullptr, LDGA_ERR_ARG, "n_iv >= 1 and n_iw >= 0 required");
    if (sp->n_iv_shell != 0)
        return ctx_fail(nullptr, LDGA_ERR_ARG, "only the plain path (n_iv_shell = 0, chi_helper = nothing) is built");
    if (precision < LDGA_PREC_FP64_INV || precision > LDGA_PREC_MIXED)
        return ctx_fail(nullptr, LDGA_ERR_ARG, "unknown precision mode");
    // G(nu) and G(nu + w) of the bubble and G(nu_n + w_n) of the EoM must lie inside fft_range
    const int need_hi = 2 * sp->n_iv + sp->n_iw - 1;
    const int need_lo = -(sp->n_iv + sp->n_iw + (sp->shift ? (sp->n_iw + 1) / 2 : 0));
    if (sp->fft_lo > need_lo || sp->fft_hi < need_hi)
        return ctx_fail(nullptr, LDGA_ERR_ARG, "fft_range too small for the frequency box");
    const int M = lat->ns / 2 + 1;
    if (!supported_grid(lat->dim, M))
        return ctx_fail(nullptr, LDGA_ERR_ARG, "k-grid size " + std::to_string(lat->ns) + " not built for dim " +
                                                   std::to_string(lat->dim));
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) return ctx_fail(nullptr, LDGA_ERR_CUDA, "no CUDA device available");
    if (device < 0 || device >= ndev) return ctx_fail(nullptr, LDGA_ERR_ARG, "device index out of range");
    ldga_ctx* c = new (std::nothrow) ldga_ctx();
    if (!c) return ctx_fail(nullptr, LDGA_ERR_ARG, "out of host memory");
    if (const char* tr = std::getenv("LDGA_TRANSFORM")) c->transform_tc = std::strcmp(tr, "tc") == 0;
    if (const char* nw = std::getenv("LDGA_NEWTON")) c->newton_async = std::strcmp(nw, "barrier") != 0;
    if (const char* dl = std::getenv("LDGA_DM_LANES")) c->dm_lanes = std::strcmp(dl, "0") != 0;
    if (const char* sw = std::getenv("LDGA_ITER_SWEEPS")) c->iter_sweeps = std::min(std::max(std::atoi(sw), 0), 1000);
    DeviceGuard g(device);
    c->device = device;
    c->newton_cluster = newton_cluster_size(c->newton_async);
    c->lat = *lat; c->mp = *mp; c->sp = *sp; c->prec = precision;
    c->dim = lat->dim; c->ns = lat->ns;
    c->Nnu = 2 * sp->n_iv; c->Nw = 2 * sp->n_iw + 1;
    c->Nf = sp->fft_hi - sp->fft_lo + 1; c->fft_lo = sp->fft_lo;
    build_kgrid(c);
    e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { g_create_error = cudaGetErrorString(e); delete c; return LDGA_ERR_CUDA; }
    c->stream = c->own_stream;
    int st = alloc_all(c);
    if (st != LDGA_OK) { g_create_error = c->err; free_all(c); cudaStreamDestroy(c->own_stream); delete c; return st; }
    *out = c;
    return LDGA_OK;
}

int ldga_destroy(ldga_ctx* ctx) {
    if (!ctx) return LDGA_OK;
    DeviceGuard g(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    free_all(ctx);
    if (ctx->graph_exec) cudaGraphExecDestroy(ctx->graph_exec);
    if (ctx->graph) cudaGraphDestroy(ctx->graph);
    if (ctx->d_chiloc) cudaFree(ctx->d_chiloc);
    if (ctx->d_gimp) cudaFree(ctx->d_gimp);
    if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
    for (auto& p : ctx->ev_pool) { cudaEventDestroy(p.a); cudaEventDestroy(p.b); }
    if (ctx->io_stream) {
        cudaStreamDestroy(ctx->io_stream);
        for (cudaEvent_t e : {ctx->ev_fork, ctx->ev_gamma, ctx->ev_loc, ctx->ev_chi, ctx->ev_join, ctx->ev_bub, ctx->ev_l0})
            if (e) cudaEventDestroy(e);
    }
    for (cudaStream_t st : ctx->dm_stream)
        if (st) cudaStreamDestroy(st);
    for (cudaEvent_t e : {ctx->dm_ev[0], ctx->dm_ev[1], ctx->dm_ev[2], ctx->dm_fork})
        if (e) cudaEventDestroy(e);
    cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return LDGA_OK;
}

int ldga_set_stream(ldga_ctx* ctx, void* stream) {
    if (!ctx) return LDGA_ERR_ARG;
    DeviceGuard g(ctx->device);
    LDGA_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
    return LDGA_OK;
}

int ldga_profile(ldga_ctx* ctx, int32_t enable) {
    if (!ctx) return LDGA_ERR_ARG;
    ctx->profiling = enable != 0;
    ctx->prof_mask = enable != 0 ? (1u << LDGA_N_STAGES) - 1u : 0u;
    return LDGA_OK;
}

int ldga_profile_stages(ldga_ctx* ctx, uint32_t mask) {
    if (!ctx) return LDGA_ERR_ARG;
    ctx->prof_mask = mask & ((1u << LDGA_N_STAGES) - 1u);
    ctx->profiling = ctx->prof_mask != 0;
    return LDGA_OK;
}

int ldga_launch_count(const ldga_ctx* ctx, int64_t* n) {
    if (!ctx || !n) return LDGA_ERR_ARG;
    *n = ctx->n_launches;
    return LDGA_OK;
}

int ldga_stage_times(ldga_ctx* ctx, double* ms, int32_t* counts) {
    if (!ctx) return LDGA_ERR_ARG;
    DeviceGuard g(ctx->device);
    LDGA_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    for (auto& pr : ctx->ev_pending) {
        float t = 0.f;
        LDGA_CUDA(ctx, cudaEventElapsedTime(&t, ctx->ev_pool[pr.second].a, ctx->ev_pool[pr.second].b));
        ctx->stage_ms[pr.first] += t;
        ctx->stage_cnt[pr.first] += 1;
        ctx->ev_free.push_back(pr.second);
    }
    ctx->ev_pending.clear();
    for (int i = 0; i < LDGA_N_STAGES; ++i) {
        if (ms) ms[i] = ctx->stage_ms[i];
        if (counts) counts[i] = ctx->stage_cnt[i];
        ctx->stage_ms[i] = 0.0;
        ctx->stage_cnt[i] = 0;
    }
    return LDGA_OK;
}

int ldga_set_model(ldga_ctx* ctx, const ldga_model* mp) {
    if (!ctx || !mp) return ctx_fail(ctx, LDGA_ERR_ARG, "null argument");
    ctx->mp = *mp;
    return LDGA_OK;
}

int ldga_set_omega_shard(ldga_ctx* ctx, int32_t w_lo, int32_t w_hi, int32_t constants) {
    if (!ctx) return LDGA_ERR_ARG;
    if (w_lo < 0 || w_hi > ctx->Nw || w_lo >= w_hi)
        return ctx_fail(ctx, LDGA_ERR_ARG, "ω shard [" + std::to_string(w_lo) + ", " + std::to_string(w_hi) +
                                               ") outside [0, " + std::to_string(ctx->Nw) + ") or empty");
    DeviceGuard g(ctx->device);
    if (w_lo != ctx->w_lo || w_hi != ctx->w_hi) {
        ctx->w_lo = w_lo;
        ctx->w_hi = w_hi;
        ctx->qperm_gen = ~0ull;   // the q order is per ω: recompute it for the new shard
        // flags outside the shard must read "solved": the fallback scans the shard's range only, but
        // a later whole-range call scans all of them
        LDGA_CUDA(ctx, cudaMemsetAsync(ctx->d_flags, 0, (size_t)ctx->Nq * ctx->Nw * sizeof(int32_t), ctx->stream));
        if (ctx->d_flags2)
            LDGA_CUDA(ctx, cudaMemsetAsync(ctx->d_flags2, 0, (size_t)ctx->Nq * ctx->Nw * sizeof(int32_t), ctx->stream));
    }
    ctx->shard_constants = constants != 0;
    return LDGA_OK;
}

int ldga_set_precision(ldga_ctx* ctx, int32_t precision) {
    if (!ctx) return LDGA_ERR_ARG;
    if (precision < LDGA_PREC_FP64_INV || precision > LDGA_PREC_MIXED)
        return ctx_fail(ctx, LDGA_ERR_ARG, "unknown precision mode");
    ctx->prec = precision;
    return LDGA_OK;
}

int ldga_kgrid(const ldga_ctx* ctx, int32_t* nk, int32_t* nq, double* kmult, double* eps, int32_t* wedge) {
    if (!ctx) return LDGA_ERR_ARG;
    if (nk) *nk = ctx->Nk;
    if (nq) *nq = ctx->Nq;
    if (kmult) std::memcpy(kmult, ctx->kmult.data(), ctx->Nq * sizeof(double));
    if (eps) std::memcpy(eps, ctx->eps.data(), ctx->Nq * sizeof(double));
    if (wedge) std::memcpy(wedge, ctx->wedge.data(), ctx->wedge.size() * sizeof(int32_t));
    return LDGA_OK;
}

int ldga_gloc(ldga_ctx* ctx, const double* sigma_loc, int32_t n_sigma, double* gloc_out) {
    if (!ctx || !sigma_loc) return ctx_fail(ctx, LDGA_ERR_ARG, "null argument");
    DeviceGuard g(ctx->device);
    TRY(set_sigma_loc(ctx, sigma_loc, n_sigma));
    TRY(launch_gloc_transform(ctx, true));
    ctx->have_ghat = true;
    if (gloc_out) TRY(copy(ctx, gloc_out, ctx->d_gloc, (size_t)ctx->Nq * ctx->Nf * sizeof(double2)));
    return sync(ctx);
}

int ldga_set_gloc(ldga_ctx* ctx, const double* gloc) {
    if (!ctx || !gloc) return ctx_fail(ctx, LDGA_ERR_ARG, "null argument");
    DeviceGuard g(ctx->device);
    TRY(copy(ctx, ctx->d_gloc, gloc, (size_t)ctx->Nq * ctx->Nf * sizeof(double2)));
    TRY(launch_gloc_transform(ctx, false));
    ctx->have_ghat = true;
    return sync(ctx);
}

int ldga_bubble(ldga_ctx* ctx, double* chi0_out) {
    if (!ctx) return LDGA_ERR_ARG;
    NEED(ctx, ctx->have_ghat, "calc_bubble: call ldga_gloc or ldga_set_gloc first");
    DeviceGuard g(ctx->device);
    TRY(launch_bubble(ctx));
    ctx->have_chi0 = true;
    if (chi0_out) TRY(copy(ctx, chi0_out, ctx->d_chi0, (size_t)ctx->Nq * ctx->Nnu * ctx->Nw * sizeof(double2)));
    return sync(ctx);
}

int ldga_set_chi0(ldga_ctx* ctx, const double* chi0) {
    if (!ctx || !chi0) return ctx_fail(ctx, LDGA_ERR_ARG, "null argument");
    DeviceGuard g(ctx->device);
    TRY(copy(ctx, ctx->d_chi0, chi0, (size_t)ctx->Nq * ctx->Nnu * ctx->Nw * sizeof(double2)));
    ++ctx->chi0_gen;
    ctx->have_chi0 = true;
    return sync(ctx);
}

int ldga_bse(ldga_ctx* ctx, int32_t channel, const double* gamma_r_in, double* chi_out, double* gam_out,
             int32_t* n_fallback) {
    if (!ctx) return LDGA_ERR_ARG;
    if (channel != LDGA_CH_M && channel != LDGA_CH_D) return ctx_fail(ctx, LDGA_ERR_TYPE, "Unkown type");
    NEED(ctx, ctx->have_chi0, "calc_χγ: bubble chi0 missing (call ldga_bubble or ldga_set_chi0)");
    DeviceGuard g(ctx->device);
    if (gamma_r_in) {
        TRY(copy(ctx, ctx->d_Gamma[channel], gamma_r_in, (size_t)ctx->Nnu * ctx->Nnu * ctx->Nw * sizeof(double2)));
        ctx->have_Gamma[channel] = true;
    }
    NEED(ctx, ctx->have_Gamma[channel], "calc_χγ: Gamma_r missing");
    LDGA_CUDA(ctx, cudaMemsetAsync(ctx->d_count, 0, 2 * sizeof(int32_t), ctx->stream));
    TRY(launch_bse(ctx, channel, ctx->d_count + 1));
    int32_t cnt[2] = {0, 0};
    TRY(copy(ctx, cnt, ctx->d_count, 2 * sizeof(int32_t)));
    TRY(sync(ctx));
    ctx->have_chi[channel] = ctx->have_gam[channel] = true;
    if (n_fallback) *n_fallback = bse_has_fast_path(ctx->Nnu) ? cnt[0] : ctx->Nq * ctx->Nw;
    if (cnt[1] > 0)
        return ctx_fail(ctx, LDGA_ERR_NUMERIC, std::to_string(cnt[1]) + " BSE matrices are singular or non-finite");
    if (chi_out) TRY(copy(ctx, chi_out, ctx->d_chi[channel], (size_t)ctx->Nq * ctx->Nw * sizeof(double)));
    if (gam_out) TRY(copy(ctx, gam_out, ctx->d_gam[channel], (size_t)ctx->Nq * ctx->Nnu * ctx->Nw * sizeof(double2)));
    return sync(ctx);
}

int ldga_bse_vjp(ldga_ctx* ctx, int32_t channel, const double* chi_bar, const double* gam_bar, double* Gamma_bar,
                 double* chi0_bar, int32_t* n_flagged) {
    if (!ctx) return LDGA_ERR_ARG;
    TRY(require_unsharded(ctx, "ldga_bse_vjp"));
    if (channel != LDGA_CH_M && channel != LDGA_CH_D) return ctx_fail(ctx, LDGA_ERR_TYPE, "Unkown type");
    NEED(ctx, ctx->have_chi0 && ctx->have_Gamma[channel] && ctx->have_chi[channel] && ctx->have_gam[channel],
         "calc_χγ adjoint: run ldga_bse for this channel first");
    DeviceGuard g(ctx->device);
    const size_t qvw = (size_t)ctx->Nq * ctx->Nnu * ctx->Nw, qw = (size_t)ctx->Nq * ctx->Nw;
    const size_t vvw = (size_t)ctx->Nnu * ctx->Nnu * ctx->Nw;
    DevScratch sc;
    double* d_xb = nullptr;
    double2 *d_gb = nullptr, *d_c0b = nullptr, *d_y = nullptr, *d_z = nullptr, *d_Gb = nullptr;
    if (chi_bar) { TRY(sc.get(ctx, &d_xb, qw)); TRY(copy(ctx, d_xb, chi_bar, qw * sizeof(double))); }
    if (gam_bar) { TRY(sc.get(ctx, &d_gb, qvw)); TRY(copy(ctx, d_gb, gam_bar, qvw * sizeof(double2))); }
    TRY(sc.get(ctx, &d_c0b, qvw));
    TRY(sc.get(ctx, &d_y, qvw));
    TRY(sc.get(ctx, &d_z, qvw));
    TRY(sc.get(ctx, &d_Gb, vvw));
    LDGA_CUDA(ctx, cudaMemsetAsync(ctx->d_count, 0, 2 * sizeof(int32_t), ctx->stream));
    TRY(launch_bse_adj(ctx, channel, d_xb, d_gb, d_c0b, d_y, d_z, d_Gb, ctx->d_count + 1));
    int32_t cnt[2] = {0, 0};
    TRY(copy(ctx, cnt, ctx->d_count, 2 * sizeof(int32_t)));
    if (Gamma_bar) TRY(copy(ctx, Gamma_bar, d_Gb, vvw * sizeof(double2)));
    if (chi0_bar) TRY(copy(ctx, chi0_bar, d_c0b, qvw * sizeof(double2)));
    TRY(sync(ctx));
    if (n_flagged) *n_flagged = cnt[1];
    return LDGA_OK;
}

int ldga_epot_vjp(ldga_ctx* ctx, int32_t numax, double mu, const double* sigma, double* sigma_bar) {
    if (!ctx || !sigma || !sigma_bar) return ctx_fail(ctx, LDGA_ERR_ARG, "null argument");
    if (numax < 1 || numax > ctx->Nnu) return ctx_fail(ctx, LDGA_ERR_ARG, "νmax out of range");
    if (!std::isfinite(mu)) return ctx_fail(ctx, LDGA_ERR_ARG, "μ must be finite");
    DeviceGuard g(ctx->device);
    const size_t n = (size_t)ctx->Nq * numax;
    DevScratch sc;
    double2 *d_s = nullptr, *d_o = nullptr;
    TRY(sc.get(ctx, &d_s, n));
    TRY(sc.get(ctx, &d_o, n));
    TRY(copy(ctx, d_s, sigma, n * sizeof(double2)));
    TRY(launch_epot_vjp(ctx, numax, mu, d_s, d_o));
    TRY(copy(ctx, sigma_bar, d_o, n * sizeof(double2)));
    return sync(ctx);
}

int ldga_autotune_bse(ldga_ctx* ctx, int32_t channel, int32_t reps, int32_t* variant, double* ms) {
    if (!ctx) return LDGA_ERR_ARG;
    if (channel != LDGA_CH_M && channel != LDGA_CH_D) return ctx_fail(ctx, LDGA_ERR_TYPE, "Unkown type");
    NEED(ctx, ctx->have_chi0 && ctx->have_Gamma[channel], "autotune: run ldga_bubble and load Gamma_r first");
    if (reps < 1) reps = 1;
    DeviceGuard g(ctx->device);
    const int nv = bse_variant_count(ctx->Nnu, ctx->prec);
    int best = 0;
    double best_ms = -1.0;
    if (nv > 1) {
        cudaEvent_t e0, e1;
        LDGA_CUDA(ctx, cudaEventCreate(&e0));
        LDGA_CUDA(ctx, cudaEventCreate(&e1));
        const bool prof = ctx->profiling;
        ctx->profiling = false;   // the trial launches stay out of the stage timers
        int st = LDGA_OK;
        auto cu = [&](cudaError_t e, const char* what) { return e == cudaSuccess ? LDGA_OK : ctx_cuda(ctx, e, what); };
        for (int i = 0; i < nv && st == LDGA_OK; ++i) {
            st = bse_run_variant(ctx, channel, i);                       // warm-up (and smem opt-in)
            if (st == LDGA_OK) st = cu(cudaEventRecord(e0, ctx->stream), "cudaEventRecord");
            for (int r = 0; r < reps && st == LDGA_OK; ++r) st = bse_run_variant(ctx, channel, i);
            if (st == LDGA_OK) st = cu(cudaEventRecord(e1, ctx->stream), "cudaEventRecord");
            if (st == LDGA_OK) st = cu(cudaEventSynchronize(e1), "cudaEventSynchronize");
            float t = 0.f;
            if (st == LDGA_OK) st = cu(cudaEventElapsedTime(&t, e0, e1), "cudaEventElapsedTime");
            const double per = (double)t / reps;
            if (st == LDGA_OK && (best_ms < 0.0 || per < best_ms)) { best_ms = per; best = i; }
        }
        ctx->profiling = prof;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (st != LDGA_OK) return st;
        bse_set_variant(ctx->Nnu, ctx->prec, best);
    }
    // leave the channel's outputs as a regular ldga_bse would (fallback for flagged matrices included)
    LDGA_CUDA(ctx, cudaMemsetAsync(ctx->d_count, 0, 2 * sizeof(int32_t), ctx->stream));
    TRY(launch_bse(ctx, channel, ctx->d_count + 1));
    int32_t cnt[2] = {0, 0};
    TRY(copy(ctx, cnt, ctx->d_count, 2 * sizeof(int32_t)));
    TRY(sync(ctx));
    ctx->have_chi[channel] = ctx->have_gam[channel] = true;
    if (variant) *variant = best;
    if (ms) *ms = best_ms;
    if (cnt[1] > 0)
        return ctx_fail(ctx, LDGA_ERR_NUMERIC, std::to_string(cnt[1]) + " BSE matrices are singular or non-finite");
    return LDGA_OK;
}

int ldga_tune_save(const char* path) {
    if (!path) return ctx_fail(nullptr, LDGA_ERR_ARG, "null path");
    FILE* f = std::fopen(path, "w");
    if (!f) return ctx_fail(nullptr, LDGA_ERR_ARG, std::string("cannot write ") + path);
    std::fprintf(f, "# libldga_b200 BSE kernel choices: bse <Nnu> <precision mode> <configuration>\n");
    for (int nnu = 1; nnu <= LDGA_MAX_NNU; ++nnu)
        for (int prec = LDGA_PREC_FP64_INV; prec <= LDGA_PREC_MIXED; ++prec) {
            const int n = bse_variant_count(nnu, prec);
            const int i = bse_tuned_variant(nnu, prec);
            if (n > 1 && i > 0 && i < n) std::fprintf(f, "bse %d %d %s\n", nnu, prec, bse_variant_name(nnu, prec, i));
        }
    std::fclose(f);
    return LDGA_OK;
}

int ldga_bse_sweeps(ldga_ctx* ctx, int64_t* passes, int64_t* warps) {
    if (!ctx) return LDGA_ERR_ARG;
    DeviceGuard g(ctx->device);
    unsigned long long v[2] = {0, 0};
    TRY(copy(ctx, v, ctx->d_iter_stats, sizeof v));
    LDGA_CUDA(ctx, cudaMemsetAsync(ctx->d_iter_stats, 0, sizeof v, ctx->stream));
    TRY(sync(ctx));
    if (passes) *passes = (int64_t)v[0];
    if (warps) *warps = (int64_t)v[1];
    return LDGA_OK;
}

const char* ldga_bse_config_name(int32_t nnu, int32_t precision, int32_t index) {
    if (index < 0) index = bse_tuned_variant(nnu, precision);
    return bse_variant_name(nnu, precision, index);
}

int ldga_tune_reset(void) {
    bse_reset_variants();
    return LDGA_OK;
}

int ldga_tune_load(const char* path) {
    if (!path) return ctx_fail(nullptr, LDGA_ERR_ARG, "null path");
    FILE* f = std::fopen(path, "r");
    if (!f) return ctx_fail(nullptr, LDGA_ERR_ARG, std::string("cannot read ") + path);
    char line[256];
    while (std::fgets(line, sizeof line, f)) {
        int nnu = 0, prec = 0;
        char name[64] = {0};
        if (std::sscanf(line, "bse %d %d %63s", &nnu, &prec, name) != 3) continue;   // comments, other lines
        const int n = bse_variant_count(nnu, prec);
        for (int i = 0; i < n; ++i)
            if (std::strcmp(bse_variant_name(nnu, prec, i), name) == 0) bse_set_variant(nnu, prec, i);
    }
    std::fclose(f);
    return LDGA_OK;
}

int ldga_get(ldga_ctx* ctx, int32_t what, int32_t channel, double* out) {
    if (!ctx || !out) return ctx_fail(ctx, LDGA_ERR_ARG, "null argument");
    DeviceGuard g(ctx->device);
    const size_t qvw = (size_t)ctx->Nq * ctx->Nnu * ctx->Nw;
    const bool ch_ok = channel == LDGA_CH_M || channel == LDGA_CH_D;
    switch (what) {
        case LDGA_GET_CHI0:
            NEED(ctx, ctx->have_chi0, "chi0 not computed");
            TRY(copy(ctx, out, ctx->d_chi0, qvw * sizeof(double2)));
            break;
        case LDGA_GET_CHI:
            if (!ch_ok) return ctx_fail(ctx, LDGA_ERR_TYPE, "Unkown type");
            NEED(ctx, ctx->have_chi[channel], "chi not computed");
            TRY(copy(ctx, out, ctx->d_chi[channel], (size_t)ctx->Nq * ctx->Nw * sizeof(double)));
            break;
        case LDGA_GET_GAMMA:
            if (!ch_ok) return ctx_fail(ctx, LDGA_ERR_TYPE, "Unkown type");
            NEED(ctx, ctx->have_gam[channel], "gamma not computed");
            TRY(copy(ctx, out, ctx->d_gam[channel], qvw * sizeof(double2)));
            break;
        case LDGA_GET_LAMBDA0:
            NEED(ctx, ctx->have_lambda0, "lambda0 not computed");
            TRY(copy(ctx, out, ctx->d_lambda0, qvw * sizeof(double2)));
            break;
        case LDGA_GET_SIGMA:
            NEED(ctx, ctx->have_sigma, "Sigma_ladder not computed");
            TRY(copy(ctx, out, ctx->d_sigma, (size_t)ctx->Nq * ctx->sigma_numax * sizeof(double2)));
            break;
        case LDGA_GET_GLOC:
            NEED(ctx, ctx->have_ghat, "G not set");
            TRY(copy(ctx, out, ctx->d_gloc, (size_t)ctx->Nq * ctx->Nf * sizeof(double2)));
            break;
        default:
            return ctx_fail(ctx, LDGA_ERR_ARG, "unknown array id");
    }
    return sync(ctx);
}

int ldga_set_chi(ldga_ctx* ctx, int32_t channel, const double* chi) {
    if (!ctx || !chi) return ctx_fail(ctx, LDGA_ERR_ARG, "null argument");
    if (channel != LDGA_CH_M && channel != LDGA_CH_D) return ctx_fail(ctx, LDGA_ERR_TYPE, "Unkown type");
    DeviceGuard g(ctx->device);
    TRY(copy(ctx, ctx->d_chi[channel], chi, (size_t)ctx->Nq * ctx->Nw * sizeof(double)));
    ctx->have_chi[channel] = true;
    return sync(ctx);
}

int ldga_set_gamma(ldga_ctx* ctx, int32_t channel, const double* gam) {
    if (!ctx || !gam) return ctx_fail(ctx, LDGA_ERR_ARG, "null argument");
    if (channel != LDGA_CH_M && channel != LDGA_CH_D) return ctx_fail(ctx, LDGA_ERR_TYPE, "Unkown type");
    DeviceGuard g(ctx->device);
    TRY(copy(ctx, ctx->d_gam[channel], gam, (size_t)ctx->Nq * ctx->Nnu * ctx->Nw * sizeof(double2)));
    ctx->have_gam[channel] = true;
    return sync(ctx);
}

int ldga_F_from_chi(ldga_ctx* ctx, const double* chi_loc, const double* gimp, int32_t n_gimp, double* F_out) {
    if (!ctx || !chi_loc || !gimp) return ctx_fail(ctx, LDGA_ERR_ARG, "null argument");
    const int need = 2 * ctx->sp.n_iv + ctx->sp.n_iw + (ctx->sp.shift ? ctx->sp.n_iw : 0);
    if (n_gimp < need) return ctx_fail(ctx, LDGA_ERR_ARG, "G_imp too short for the frequency box");
    DeviceGuard g(ctx->device);
    const size_t nF = (size_t)ctx->Nnu * ctx->Nnu * ctx->Nw;
    double2* d_chi = nullptr;
    double2* d_g = nullptr;
    LDGA_CUDA(ctx, cudaMallocAsync(reinterpret_cast<void**>(&d_chi), nF * sizeof(double2), ctx->stream));
    LDGA_CUDA(ctx, cudaMallocAsync(reinterpret_cast<void**>(&d_g), (size_t)n_gimp * sizeof(double2), ctx->stream));
    int st = copy(ctx, d_chi, chi_loc, nF * sizeof(double2));
    if (!st) st = copy(ctx, d_g, gimp, (size_t)n_gimp * sizeof(double2));
    if (!st) st = launch_F_from_chi(ctx, d_chi, d_g, n_gimp);
    cudaFreeAsync(d_chi, ctx->stream);
    cudaFreeAsync(d_g, ctx->stream);
    TRY(st);
    ctx->have_F = true;
    if (F_out) TRY(copy(ctx, F_out, ctx->d_F, nF * sizeof(double2)));
    return sync(ctx);
}

int ldga_lambda0(ldga_ctx* ctx, const double* F_in, double* lambda0_out) {
    if (!ctx) return LDGA_ERR_ARG;
    NEED(ctx, ctx->have_chi0, "calc_λ0: bubble chi0 missing");
    DeviceGuard g(ctx->device);
    const size_t nF = (size_t)ctx->Nnu * ctx->Nnu * ctx->Nw;
    if (F_in) { TRY(copy(ctx, ctx->d_F, F_in, nF * sizeof(double2))); ctx->have_F = true; }
    NEED(ctx, ctx->have_F, "calc_λ0: F missing (call ldga_F_from_chi or pass F)");
    TRY(launch_lambda0(ctx));
    ctx->have_lambda0 = true;
    if (lambda0_out) TRY(copy(ctx, lambda0_out, ctx->d_lambda0, (size_t)ctx->Nq * ctx->Nnu * ctx->Nw * sizeof(double2)));
    return sync(ctx);
}

int ldga_set_lambda0(ldga_ctx* ctx, const double* lambda0) {
    if (!ctx || !lambda0) return ctx_fail(ctx, LDGA_ERR_ARG, "null argument");
    DeviceGuard g(ctx->device);
    TRY(copy(ctx, ctx->d_lambda0, lambda0, (size_t)ctx->Nq * ctx->Nnu * ctx->Nw * sizeof(double2)));
    ctx->have_lambda0 = true;
    return sync(ctx);
}

int ldga_sum_kw(ldga_ctx* ctx, int32_t channel, double lam, int32_t deriv, double* out) {
    if (!ctx || !out) return ctx_fail(ctx, LDGA_ERR_ARG, "null argument");
    if (channel != LDGA_CH_M && channel != LDGA_CH_D) return ctx_fail(ctx, LDGA_ERR_TYPE, "Unkown type");
    NEED(ctx, ctx->have_chi[channel], "sum_kω: chi missing");
    DeviceGuard g(ctx->device);
    TRY(launch_sum_kw(ctx, channel, lam, deriv ? 1 : 0, ctx->d_red));
    TRY(copy(ctx, out, ctx->d_red, sizeof(double)));
    return sync(ctx);
}

int ldga_sum_wk(ldga_ctx* ctx, int32_t channel, double lam, double* out) {
    if (!ctx || !out) return ctx_fail(ctx, LDGA_ERR_ARG, "null argument");
    if (channel != LDGA_CH_M && channel != LDGA_CH_D) return ctx_fail(ctx, LDGA_ERR_TYPE, "Unkown type");
    NEED(ctx, ctx->have_chi[channel], "sum_ωk: chi missing");
    DeviceGuard g(ctx->device);
    TRY(launch_sum_kw(ctx, channel, lam, 2, ctx->d_red));
    TRY(copy(ctx, out, ctx->d_red, sizeof(double)));
    return sync(ctx);
}

int ldga_lambda_min(ldga_ctx* ctx, int32_t channel, double* out) {
    if (!ctx || !out) return ctx_fail(ctx, LDGA_ERR_ARG, "null argument");
    if (channel != LDGA_CH_M && channel != LDGA_CH_D) return ctx_fail(ctx, LDGA_ERR_TYPE, "Unkown type");
    NEED(ctx, ctx->have_chi[channel], "get_λ_min: chi missing");
    DeviceGuard g(ctx->device);
    TRY(launch_lambda_min(ctx, channel, ctx->d_red));
    TRY(copy(ctx, out, ctx->d_red, sizeof(double)));
    return sync(ctx);
}

namespace {
int eom_inputs_ready(ldga_ctx* ctx) {
    NEED(ctx, ctx->have_ghat, "calc_Σ: G transform missing");
    NEED(ctx, ctx->have_chi[0] && ctx->have_chi[1], "calc_Σ: chi_m / chi_d missing");
    NEED(ctx, ctx->have_gam[0] && ctx->have_gam[1], "calc_Σ: gamma_m / gamma_d missing");
    NEED(ctx, ctx->have_lambda0, "calc_Σ: lambda0 missing");
    return LDGA_OK;
}

// EoM into d_sigma (all on the stream, no sync)
// tail_dev: device scalar sum_kω(χ_m^λm) formed earlier on the stream (the EoM tail's); null: formed
// here into d_red[8]
int eom_device(ldga_ctx* ctx, double lam_m, double lam_d, int numax, int tc, double chiloc_m_sum,
               const double* tail_dev = nullptr) {
    if (numax < 1 || numax > ctx->Nnu) return ctx_fail(ctx, LDGA_ERR_ARG, "νmax out of range");
    if (numax > std::abs(ctx->fft_lo) - ctx->sp.n_iw) return ctx_fail(ctx, LDGA_ERR_ARG, "νmax exceeds fft_range");
    if (tc && !tail_dev) TRY(launch_sum_kw(ctx, LDGA_CH_M, lam_m, 0, ctx->d_red + 8));
    TRY(launch_eom(ctx, numax, lam_m, lam_d, nullptr, nullptr, -1, tail_dev ? tail_dev : ctx->d_red + 8, tc,
                   chiloc_m_sum, ctx->d_sigma, ctx->Nq, 1));
    ctx->have_sigma = true;
    ctx->sigma_numax = numax;
    return LDGA_OK;
}
}  // namespace

int ldga_eom(ldga_ctx* ctx, double lam_m, double lam_d, int32_t numax, int32_t tc, double chiloc_m_sum,
             double* sigma_out) {
    if (!ctx) return LDGA_ERR_ARG;
    TRY(eom_inputs_ready(ctx));
    if (!std::isfinite(lam_m) || !std::isfinite(lam_d)) return ctx_fail(ctx, LDGA_ERR_ARG, "λ must be finite");
    DeviceGuard g(ctx->device);
    TRY(eom_device(ctx, lam_m, lam_d, numax, tc, chiloc_m_sum));
    if (sigma_out) TRY(copy(ctx, sigma_out, ctx->d_sigma, (size_t)ctx->Nq * numax * sizeof(double2)));
    return sync(ctx);
}

int ldga_eom_vjp(ldga_ctx* ctx, double lam_m, double lam_d, int32_t numax, int32_t tc, const double* sigma_bar,
                 double* chi_m_bar, double* gam_m_bar, double* chi_d_bar, double* gam_d_bar, double* lambda0_bar) {
    if (!ctx || !sigma_bar) return ctx_fail(ctx, LDGA_ERR_ARG, "null argument");
    TRY(require_unsharded(ctx, "ldga_eom_vjp"));
    TRY(eom_inputs_ready(ctx));
    if (!std::isfinite(lam_m) || !std::isfinite(lam_d)) return ctx_fail(ctx, LDGA_ERR_ARG, "λ must be finite");
    if (numax < 1 || numax > ctx->Nnu) return ctx_fail(ctx, LDGA_ERR_ARG, "νmax out of range");
    if (numax > std::abs(ctx->fft_lo) - ctx->sp.n_iw) return ctx_fail(ctx, LDGA_ERR_ARG, "νmax exceeds fft_range");
    DeviceGuard g(ctx->device);
    const size_t qvw = (size_t)ctx->Nq * ctx->Nnu * ctx->Nw, qw = (size_t)ctx->Nq * ctx->Nw;
    const size_t nsb = (size_t)ctx->Nq * numax;
    DevScratch sc;
    double2 *d_sb = nullptr, *d_shat = nullptr, *d_gm = nullptr, *d_gd = nullptr, *d_l0 = nullptr;
    double *d_xm = nullptr, *d_xd = nullptr, *d_cm = nullptr, *d_cd = nullptr;
    TRY(sc.get(ctx, &d_sb, nsb));
    TRY(copy(ctx, d_sb, sigma_bar, nsb * sizeof(double2)));
    TRY(sc.get(ctx, &d_shat, nsb));
    TRY(sc.get(ctx, &d_cm, nsb * ctx->Nw));
    TRY(sc.get(ctx, &d_cd, nsb * ctx->Nw));
    if (gam_m_bar) { TRY(sc.get(ctx, &d_gm, qvw)); LDGA_CUDA(ctx, cudaMemsetAsync(d_gm, 0, qvw * sizeof(double2), ctx->stream)); }
    if (gam_d_bar) { TRY(sc.get(ctx, &d_gd, qvw)); LDGA_CUDA(ctx, cudaMemsetAsync(d_gd, 0, qvw * sizeof(double2), ctx->stream)); }
    if (lambda0_bar) { TRY(sc.get(ctx, &d_l0, qvw)); LDGA_CUDA(ctx, cudaMemsetAsync(d_l0, 0, qvw * sizeof(double2), ctx->stream)); }
    if (chi_m_bar) TRY(sc.get(ctx, &d_xm, qw));
    if (chi_d_bar) TRY(sc.get(ctx, &d_xd, qw));
    TRY(launch_eom_vjp(ctx, numax, lam_m, lam_d, tc, d_sb, d_gm, d_gd, d_l0, d_xm, d_xd, d_shat, d_cm, d_cd));
    if (gam_m_bar) TRY(copy(ctx, gam_m_bar, d_gm, qvw * sizeof(double2)));
    if (gam_d_bar) TRY(copy(ctx, gam_d_bar, d_gd, qvw * sizeof(double2)));
    if (lambda0_bar) TRY(copy(ctx, lambda0_bar, d_l0, qvw * sizeof(double2)));
    if (chi_m_bar) TRY(copy(ctx, chi_m_bar, d_xm, qw * sizeof(double)));
    if (chi_d_bar) TRY(copy(ctx, chi_d_bar, d_xd, qw * sizeof(double)));
    return sync(ctx);
}

int ldga_gloc_vjp(ldga_ctx* ctx, const double* chi0_bar, const double* lambda0_bar, const double* sigma_bar,
                  double lam_m, double lam_d, int32_t numax, int32_t n_sigma, double* sigma_loc_bar, double* gloc_bar) {
    if (!ctx) return LDGA_ERR_ARG;
    TRY(require_unsharded(ctx, "ldga_gloc_vjp"));
    NEED(ctx, ctx->have_ghat, "G adjoint: call ldga_gloc first");
    if (lambda0_bar) NEED(ctx, ctx->have_F, "G adjoint: F_m missing (call ldga_F_from_chi)");
    if (sigma_bar) {
        TRY(eom_inputs_ready(ctx));
        if (numax < 1 || numax > ctx->Nnu) return ctx_fail(ctx, LDGA_ERR_ARG, "νmax out of range");
        if (numax > std::abs(ctx->fft_lo) - ctx->sp.n_iw) return ctx_fail(ctx, LDGA_ERR_ARG, "νmax exceeds fft_range");
    } else {
        numax = 0;
    }
    if (sigma_loc_bar && n_sigma < 1) return ctx_fail(ctx, LDGA_ERR_ARG, "n_sigma must be >= 1");
    DeviceGuard g(ctx->device);
    const size_t qvw = (size_t)ctx->Nq * ctx->Nnu * ctx->Nw, nfq = (size_t)ctx->Nf * ctx->Nq;
    const bool bub = chi0_bar || lambda0_bar;
    DevScratch sc;
    double2 *d_c0b = nullptr, *d_l0b = nullptr, *d_sb = nullptr, *d_slb = nullptr, *d_gb = nullptr;
    if (bub) {
        TRY(sc.get(ctx, &d_c0b, qvw));
        if (chi0_bar) TRY(copy(ctx, d_c0b, chi0_bar, qvw * sizeof(double2)));
        else LDGA_CUDA(ctx, cudaMemsetAsync(d_c0b, 0, qvw * sizeof(double2), ctx->stream));
        if (lambda0_bar) {
            TRY(sc.get(ctx, &d_l0b, qvw));
            TRY(copy(ctx, d_l0b, lambda0_bar, qvw * sizeof(double2)));
            TRY(launch_lambda0_vjp(ctx, d_l0b, d_c0b));
        }
    }
    if (numax > 0) {
        TRY(sc.get(ctx, &d_sb, (size_t)ctx->Nq * numax));
        TRY(copy(ctx, d_sb, sigma_bar, (size_t)ctx->Nq * numax * sizeof(double2)));
    }
    std::vector<int32_t> start, idx;
    TRY(gloc_vjp_device(ctx, sc, d_c0b, d_sb, numax, lam_m, lam_d, sigma_loc_bar ? n_sigma : 0, start, idx, &d_slb,
                        &d_gb));
    if (sigma_loc_bar) TRY(copy(ctx, sigma_loc_bar, d_slb, (size_t)n_sigma * sizeof(double2)));
    if (gloc_bar) TRY(copy(ctx, gloc_bar, d_gb, nfq * sizeof(double2)));
    return sync(ctx);   // host vectors (start, idx) outlive the asynchronous copies
}

int ldga_chain_vjp(ldga_ctx* ctx, const double* sigma_bar, double lam_m, double lam_d, int32_t numax, int32_t tc,
                   double* Gamma_m_bar, double* Gamma_d_bar, int32_t n_sigma, double* sigma_loc_bar,
                   double* chi0_bar, int32_t* n_flagged) {
    if (!ctx || !sigma_bar) return ctx_fail(ctx, LDGA_ERR_ARG, "null argument");
    TRY(require_unsharded(ctx, "ldga_chain_vjp"));
    TRY(eom_inputs_ready(ctx));
    NEED(ctx, ctx->have_chi0 && ctx->have_Gamma[0] && ctx->have_Gamma[1],
         "chain adjoint: run the bubble and both BSE channels first");
    NEED(ctx, ctx->have_F, "chain adjoint: F_m missing (call ldga_F_from_chi)");
    if (!std::isfinite(lam_m) || !std::isfinite(lam_d)) return ctx_fail(ctx, LDGA_ERR_ARG, "λ must be finite");
    if (numax < 1 || numax > ctx->Nnu) return ctx_fail(ctx, LDGA_ERR_ARG, "νmax out of range");
    if (numax > std::abs(ctx->fft_lo) - ctx->sp.n_iw) return ctx_fail(ctx, LDGA_ERR_ARG, "νmax exceeds fft_range");
    if (sigma_loc_bar && n_sigma < 1) return ctx_fail(ctx, LDGA_ERR_ARG, "n_sigma must be >= 1");
    DeviceGuard g(ctx->device);
    const size_t qvw = (size_t)ctx->Nq * ctx->Nnu * ctx->Nw, qw = (size_t)ctx->Nq * ctx->Nw;
    const size_t vvw = (size_t)ctx->Nnu * ctx->Nnu * ctx->Nw, nsb = (size_t)ctx->Nq * numax;
    DevScratch sc;
    double2 *d_sb = nullptr, *d_shat = nullptr, *d_gm = nullptr, *d_gd = nullptr, *d_l0 = nullptr;
    double *d_xm = nullptr, *d_xd = nullptr, *d_cm = nullptr, *d_cd = nullptr;
    double2 *d_c0b = nullptr, *d_y = nullptr, *d_z = nullptr, *d_Gm = nullptr, *d_Gd = nullptr;
    double2 *d_slb = nullptr, *d_gb = nullptr;
    // 1. EoM: Sigma_bar -> gamma_m_bar, gamma_d_bar, lambda0_bar, chi_m_bar, chi_d_bar
    TRY(sc.get(ctx, &d_sb, nsb));
    TRY(copy(ctx, d_sb, sigma_bar, nsb * sizeof(double2)));
    TRY(sc.get(ctx, &d_shat, nsb));
    TRY(sc.get(ctx, &d_cm, nsb * ctx->Nw));
    TRY(sc.get(ctx, &d_cd, nsb * ctx->Nw));
    TRY(sc.get(ctx, &d_gm, qvw));
    TRY(sc.get(ctx, &d_gd, qvw));
    TRY(sc.get(ctx, &d_l0, qvw));
    TRY(sc.get(ctx, &d_xm, qw));
    TRY(sc.get(ctx, &d_xd, qw));
    LDGA_CUDA(ctx, cudaMemsetAsync(d_gm, 0, qvw * sizeof(double2), ctx->stream));
    LDGA_CUDA(ctx, cudaMemsetAsync(d_gd, 0, qvw * sizeof(double2), ctx->stream));
    LDGA_CUDA(ctx, cudaMemsetAsync(d_l0, 0, qvw * sizeof(double2), ctx->stream));
    TRY(launch_eom_vjp(ctx, numax, lam_m, lam_d, tc, d_sb, d_gm, d_gd, d_l0, d_xm, d_xd, d_shat, d_cm, d_cd));
    // 2. both BSE channels -> Gamma_bar_r, chi0_bar (summed), then lambda0 -> chi0_bar
    TRY(sc.get(ctx, &d_c0b, qvw));
    TRY(sc.get(ctx, &d_y, qvw));
    TRY(sc.get(ctx, &d_z, qvw));
    TRY(sc.get(ctx, &d_Gm, vvw));
    TRY(sc.get(ctx, &d_Gd, vvw));
    LDGA_CUDA(ctx, cudaMemsetAsync(ctx->d_count, 0, 2 * sizeof(int32_t), ctx->stream));
    TRY(launch_bse_adj(ctx, LDGA_CH_M, d_xm, d_gm, d_c0b, d_y, d_z, d_Gm, ctx->d_count + 1, false));
    TRY(launch_bse_adj(ctx, LDGA_CH_D, d_xd, d_gd, d_c0b, d_y, d_z, d_Gd, ctx->d_count + 1, true));
    TRY(launch_lambda0_vjp(ctx, d_l0, d_c0b));
    // 3. lattice G: bubble (chi0_bar) and the EoM's G (Sigma_bar) -> G_bar -> Sigma_loc_bar
    std::vector<int32_t> start, idx;
    if (sigma_loc_bar)
        TRY(gloc_vjp_device(ctx, sc, d_c0b, d_sb, numax, lam_m, lam_d, n_sigma, start, idx, &d_slb, &d_gb));
    int32_t cnt[2] = {0, 0};
    TRY(copy(ctx, cnt, ctx->d_count, 2 * sizeof(int32_t)));
    if (Gamma_m_bar) TRY(copy(ctx, Gamma_m_bar, d_Gm, vvw * sizeof(double2)));
    if (Gamma_d_bar) TRY(copy(ctx, Gamma_d_bar, d_Gd, vvw * sizeof(double2)));
    if (chi0_bar) TRY(copy(ctx, chi0_bar, d_c0b, qvw * sizeof(double2)));
    if (sigma_loc_bar) TRY(copy(ctx, sigma_loc_bar, d_slb, (size_t)n_sigma * sizeof(double2)));
    TRY(sync(ctx));
    if (n_flagged) *n_flagged = cnt[1];
    return LDGA_OK;
}

int ldga_eom_parts(ldga_ctx* ctx, double lam_m, double lam_d, int32_t tc, double chiloc_m_sum, double* parts_out) {
    if (!ctx || !parts_out) return ctx_fail(ctx, LDGA_ERR_ARG, "null argument");
    TRY(require_unsharded(ctx, "ldga_eom_parts"));
    TRY(eom_inputs_ready(ctx));
    DeviceGuard g(ctx->device);
    const int numax = ctx->sp.n_iv;
    const size_t blk = (size_t)ctx->Nq * numax;
    double2* d_parts = nullptr;
    LDGA_CUDA(ctx, cudaMallocAsync(reinterpret_cast<void**>(&d_parts), 7 * blk * sizeof(double2), ctx->stream));
    int st = LDGA_OK;
    for (int p = 0; p < 6 && st == LDGA_OK; ++p)
        st = launch_eom(ctx, numax, lam_m, lam_d, nullptr, nullptr, p, ctx->d_red, 0, 0.0, d_parts + p * blk, ctx->Nq,
                        p == 5 ? 1 : 0);
    double tnum = 0.0;
    if (st == LDGA_OK && tc) {
        st = launch_sum_kw(ctx, LDGA_CH_M, lam_m, 0, ctx->d_red + 8);
        double s = 0.0;
        if (st == LDGA_OK) st = copy(ctx, &s, ctx->d_red + 8, sizeof(double));
        if (st == LDGA_OK) st = sync(ctx);
        tnum = -ctx->mp.U * (s - chiloc_m_sum);
    }
    if (st == LDGA_OK) st = launch_fill_tail(ctx, numax, tnum, d_parts + 6 * blk, ctx->Nq);
    if (st == LDGA_OK) st = copy(ctx, parts_out, d_parts, 7 * blk * sizeof(double2));
    cudaFreeAsync(d_parts, ctx->stream);
    TRY(st);
    return sync(ctx);
}

int ldga_lambda_m_newton(ldga_ctx* ctx, double rhs, int32_t nsteps, double atol, double* lam_out,
                         int32_t* iterations, int32_t* period) {
    if (!ctx || !lam_out) return ctx_fail(ctx, LDGA_ERR_ARG, "null argument");
    if (nsteps < 1 || !(atol >= 0.0)) return ctx_fail(ctx, LDGA_ERR_ARG, "newton_right: nsteps >= 1, atol >= 0");
    NEED(ctx, ctx->have_chi[LDGA_CH_M], "λm_correction: chi_m missing");
    DeviceGuard g(ctx->device);
    TRY(launch_lambda_m(ctx, rhs, nullptr, ctx->d_red + 16, nsteps, atol));
    double r[5];
    TRY(copy(ctx, r, ctx->d_red + 16, 5 * sizeof(double)));
    TRY(sync(ctx));
    *lam_out = r[0];
    if (iterations) *iterations = (int32_t)r[1];
    if (period) { period[0] = (int32_t)r[3]; period[1] = (int32_t)r[4]; }
    return LDGA_OK;
}

int ldga_lambda_m(ldga_ctx* ctx, double rhs, double* lam_out, int32_t* iterations) {
    return ldga_lambda_m_newton(ctx, rhs, 100, 1e-13, lam_out, iterations, nullptr);
}

int ldga_g_ladder(ldga_ctx* ctx, const double* sigma_loc, int32_t n_sigma, int32_t fix_n, double mu_in,
                  double* mu_out, double* G_out, double* e_kin, double* e_pot, double* n_out) {
    if (!ctx) return LDGA_ERR_ARG;
    NEED(ctx, ctx->have_sigma, "G_from_Σladder: no Sigma_ladder on the device (call ldga_eom)");
    DeviceGuard g(ctx->device);
    if (sigma_loc) TRY(set_sigma_loc(ctx, sigma_loc, n_sigma));
    NEED(ctx, ctx->d_sigma_loc != nullptr, "G_from_Σladder: Sigma_loc missing");
    TRY(launch_g_ladder(ctx, ctx->sigma_numax, fix_n, mu_in, ctx->d_red + 24));
    double r[4];
    TRY(copy(ctx, r, ctx->d_red + 24, 4 * sizeof(double)));
    TRY(sync(ctx));
    if (G_out) {
        TRY(launch_g_ladder_full(ctx, ctx->sigma_numax, ctx->d_red + 24));
        TRY(copy(ctx, G_out, ctx->d_gladder, (size_t)ctx->Nq * ctx->Nf * sizeof(double2)));
        TRY(sync(ctx));
    }
    if (mu_out) *mu_out = r[0];
    if (e_kin) *e_kin = r[1];
    if (e_pot) *e_pot = r[2];
    if (n_out) *n_out = r[3];
    if (!std::isfinite(r[0])) return ctx_fail(ctx, LDGA_ERR_NOCONV, "μ determination failed");
    return LDGA_OK;
}

int ldga_set_sigma(ldga_ctx* ctx, const double* sigma, int32_t numax) {
    if (!ctx || !sigma) return ctx_fail(ctx, LDGA_ERR_ARG, "null argument");
    if (numax < 1 || numax > ctx->Nnu) return ctx_fail(ctx, LDGA_ERR_ARG, "νmax out of range");
    DeviceGuard g(ctx->device);
    TRY(copy(ctx, ctx->d_sigma, sigma, (size_t)ctx->Nq * numax * sizeof(double2)));
    ctx->have_sigma = true;
    ctx->sigma_numax = numax;
    return sync(ctx);
}

int ldga_calc_E(ldga_ctx* ctx, const double* G, const double* sigma, int32_t numax, double mu, double* e_kin,
                double* e_pot) {
    if (!ctx) return LDGA_ERR_ARG;
    if (numax < 1 || numax > ctx->Nnu) return ctx_fail(ctx, LDGA_ERR_ARG, "νmax out of range");
    DeviceGuard g(ctx->device);
    const size_t blk = (size_t)ctx->Nq * numax;
    double2* d_tmp = nullptr;
    const double2* dG = nullptr;
    const double2* dS = ctx->d_sigma;
    int ldg = ctx->Nq;
    if (G || sigma) LDGA_CUDA(ctx, cudaMallocAsync(reinterpret_cast<void**>(&d_tmp), 2 * blk * sizeof(double2), ctx->stream));
    int st = LDGA_OK;
    if (G) { st = copy(ctx, d_tmp, G, blk * sizeof(double2)); dG = d_tmp; }
    else { dG = ctx->d_gladder - ctx->fft_lo * (ptrdiff_t)ctx->Nq; }   // column nu_n = 0 of G_ladder
    if (!st && sigma) { st = copy(ctx, d_tmp + blk, sigma, blk * sizeof(double2)); dS = d_tmp + blk; }
    if (!st) st = launch_calc_E(ctx, dG, ldg, dS, numax, mu, ctx->d_red + 48);
    double r[2] = {0.0, 0.0};
    if (!st) st = copy(ctx, r, ctx->d_red + 48, 2 * sizeof(double));
    if (d_tmp) cudaFreeAsync(d_tmp, ctx->stream);
    TRY(st);
    TRY(sync(ctx));
    if (e_kin) *e_kin = r[0];
    if (e_pot) *e_pot = r[1];
    return LDGA_OK;
}

// -------------------------------------------------------------------------- fused lambda_m chain --
namespace {

bool host_pageable(const void* p) {
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) { cudaGetLastError(); return true; }
    return a.type == cudaMemoryTypeUnregistered;
}

struct ChainArgs {
    const double *sigma_loc, *gamma_m, *gamma_d, *chi_loc_m, *gimp;
    int n_sigma, n_gimp;
    double imp_density, chiloc_m_sum;
    double *sigma_out, *chi_m_out, *chi_d_out;
};

// Enqueue the whole chain on ctx->stream; nothing here waits for the device.  The inputs the first
// stages do not need (Γ_m, Γ_d, χ_loc,m, G_imp) are copied on io_stream while the G transform and the
// bubble run, and χ_m, χ_d are copied out there while the λ and EoM stages run; the main stream waits
// for each copy through an event before its first use and for all of them at the end (under capture
// the events become graph edges).
int chain_m_enqueue(ldga_ctx* ctx, const ChainArgs& a) {
    const size_t nG = (size_t)ctx->Nnu * ctx->Nnu * ctx->Nw * sizeof(double2);
    const size_t nX = (size_t)ctx->Nq * ctx->Nw * sizeof(double);
    const int numax = ctx->Nnu / 2;
    cudaStream_t io = ctx->io_stream;
    auto cp = [&](void* dst, const void* src, size_t bytes) -> int {
        LDGA_CUDA(ctx, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, io));
        return LDGA_OK;
    };
    LDGA_CUDA(ctx, cudaEventRecord(ctx->ev_fork, ctx->stream));
    LDGA_CUDA(ctx, cudaStreamWaitEvent(io, ctx->ev_fork, 0));
    TRY(cp(ctx->d_Gamma[0], a.gamma_m, nG));
    TRY(cp(ctx->d_Gamma[1], a.gamma_d, nG));
    LDGA_CUDA(ctx, cudaEventRecord(ctx->ev_gamma, io));
    TRY(cp(ctx->d_chiloc, a.chi_loc_m, nG));
    TRY(cp(ctx->d_gimp, a.gimp, (size_t)a.n_gimp * sizeof(double2)));
    LDGA_CUDA(ctx, cudaEventRecord(ctx->ev_loc, io));
    TRY(copy(ctx, ctx->d_sigma_loc, a.sigma_loc, (size_t)a.n_sigma * sizeof(double2)));
    TRY(launch_gloc_transform(ctx, true));                       // a1
    TRY(launch_bubble(ctx));                                     // a2
    // a5, a6 need χ₀ and the local inputs only.  A chain alone on the GPU runs them on the copy
    // stream beside the BSE and the λm Newton (16 SMs), and the EoM waits for them; their scratch
    // (d_red from 64 on) is theirs.  Chains of a batch (l0_beside false) keep them on their main
    // stream: with many chains side by side the GPU has no idle SMs to give them, and the batch ran
    // 37.8 ms with them in line against 43.8 ms beside.
    if (ctx->l0_beside) {
        LDGA_CUDA(ctx, cudaEventRecord(ctx->ev_bub, ctx->stream));
        LDGA_CUDA(ctx, cudaStreamWaitEvent(io, ctx->ev_bub, 0));
        cudaStream_t main = ctx->stream;
        ctx->stream = io;
        const int st = launch_F_from_chi(ctx, ctx->d_chiloc, ctx->d_gimp, a.n_gimp);   // a5
        const int st2 = st == LDGA_OK ? launch_lambda0(ctx) : st;                      // a6
        ctx->stream = main;
        TRY(st2);
        LDGA_CUDA(ctx, cudaEventRecord(ctx->ev_l0, io));
    } else {
        LDGA_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->ev_loc, 0));
        TRY(launch_F_from_chi(ctx, ctx->d_chiloc, ctx->d_gimp, a.n_gimp));   // a5
        TRY(launch_lambda0(ctx));                                           // a6
    }
    LDGA_CUDA(ctx, cudaMemsetAsync(ctx->d_count, 0, 4 * sizeof(int32_t), ctx->stream));   // fails, lists
    LDGA_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->ev_gamma, 0));
    TRY(launch_bse_pair(ctx, ctx->d_count + 1));                  // a7, both channels
    LDGA_CUDA(ctx, cudaEventRecord(ctx->ev_chi, ctx->stream));
    LDGA_CUDA(ctx, cudaStreamWaitEvent(io, ctx->ev_chi, 0));
    if (a.chi_m_out) TRY(cp(a.chi_m_out, ctx->d_chi[0], nX));
    if (a.chi_d_out) TRY(cp(a.chi_d_out, ctx->d_chi[1], nX));
    LDGA_CUDA(ctx, cudaEventRecord(ctx->ev_join, io));
    // λm_correction_full (conditions_new.jl:174-190): rhs = 2 imp_density - sum_kω(chi_d), the Newton, and
    // sum_kω(chi_m, λ = λm) for the EoM's tail, all in the Newton kernel (d_red[56], d_red[16], d_red[8])
    TRY(launch_lambda_m(ctx, 2.0 * a.imp_density, nullptr, ctx->d_red + 16, 100, 1e-13, ctx->d_red + 56,
                        ctx->d_red + 8));
    if (ctx->l0_beside) LDGA_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->ev_l0, 0));
    TRY(launch_eom(ctx, numax, 0.0, 0.0, ctx->d_red + 16, nullptr, -1, ctx->d_red + 8, 1, a.chiloc_m_sum,
                   ctx->d_sigma, ctx->Nq, 1));                   // a10 at λm
    TRY(launch_g_ladder(ctx, numax, 1, ctx->mp.mu, ctx->d_red + 24));   // a15: μ fit, energies
    if (a.sigma_out) TRY(copy(ctx, a.sigma_out, ctx->d_sigma, (size_t)ctx->Nq * numax * sizeof(double2)));
    TRY(copy(ctx, ctx->h_stage, ctx->d_red, 64 * sizeof(double)));
    TRY(copy(ctx, ctx->h_stage + 64, ctx->d_count, 4 * sizeof(int32_t)));
    LDGA_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->ev_join, 0));
    return LDGA_OK;
}

uint64_t dbits(double x) { uint64_t u; std::memcpy(&u, &x, 8); return u; }

}  // namespace

namespace {

// Checks the inputs, allocates the chain's persistent buffers and enqueues the chain on the handle's
// stream: a replay of the captured graph when pointers and scalars are unchanged, otherwise an
// uncaptured run (it computes this call's results) followed by a capture.  Nothing waits for the
// device, so several handles' chains can be in flight at once.
int chain_m_submit(ldga_ctx* ctx, const ChainArgs& a, bool use_graph, bool* replayed_out) {
    *replayed_out = false;
    if (!a.sigma_loc || !a.gamma_m || !a.gamma_d || !a.chi_loc_m || !a.gimp)
        return ctx_fail(ctx, LDGA_ERR_ARG, "null argument");
    const int n_sigma = a.n_sigma, n_gimp = a.n_gimp;
    const int L = std::max(std::abs(ctx->sp.fft_lo), std::abs(ctx->sp.fft_hi));
    if (n_sigma <= L) return ctx_fail(ctx, LDGA_ERR_ARG, "Sigma_loc must cover n = 0..max|fft_range|");
    const int need_g = 2 * ctx->sp.n_iv + ctx->sp.n_iw + (ctx->sp.shift ? ctx->sp.n_iw : 0);
    if (n_gimp < need_g) return ctx_fail(ctx, LDGA_ERR_ARG, "G_imp too short for the frequency box");
    // buffers (allocated outside any capture)
    if (n_sigma > ctx->n_sigma_loc) {
        if (ctx->d_sigma_loc) cudaFree(ctx->d_sigma_loc);
        ctx->d_sigma_loc = nullptr;
        TRY(dev_alloc(ctx, &ctx->d_sigma_loc, (size_t)n_sigma));
        ctx->n_sigma_loc = n_sigma;
    }
    ctx->n_sigma_loc = std::max(ctx->n_sigma_loc, (int)n_sigma);
    TRY(dev_alloc(ctx, &ctx->d_chiloc, (size_t)ctx->Nnu * ctx->Nnu * ctx->Nw));
    if (n_gimp > ctx->n_gimp_alloc) {
        if (ctx->d_gimp) cudaFree(ctx->d_gimp);
        ctx->d_gimp = nullptr;
        TRY(dev_alloc(ctx, &ctx->d_gimp, (size_t)n_gimp));
        ctx->n_gimp_alloc = n_gimp;
    }
    if (!ctx->h_stage) LDGA_CUDA(ctx, cudaMallocHost(reinterpret_cast<void**>(&ctx->h_stage), 64 * sizeof(double) + 16));
    if (!ctx->io_stream) {
        LDGA_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->io_stream, cudaStreamNonBlocking));
        for (cudaEvent_t* e : {&ctx->ev_fork, &ctx->ev_gamma, &ctx->ev_loc, &ctx->ev_chi, &ctx->ev_join, &ctx->ev_bub,
                               &ctx->ev_l0})
            LDGA_CUDA(ctx, cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    }
    const void* ptrs[] = {a.sigma_loc, a.gamma_m, a.gamma_d, a.chi_loc_m, a.gimp, a.sigma_out, a.chi_m_out, a.chi_d_out};
    bool graphable = use_graph;
    for (const void* p : ptrs)
        if (host_pageable(p)) graphable = false;   // stream capture needs pinned or device memory
    std::vector<uint64_t> key;
    if (graphable) {
        for (const void* p : ptrs) key.push_back((uint64_t)(uintptr_t)p);
        key.insert(key.end(), {(uint64_t)n_sigma, (uint64_t)n_gimp, dbits(a.imp_density), dbits(a.chiloc_m_sum),
                               dbits(ctx->mp.U), dbits(ctx->mp.mu), dbits(ctx->mp.beta), dbits(ctx->mp.n),
                               dbits(ctx->mp.Ekin_DMFT), (uint64_t)ctx->prec, (uint64_t)(uintptr_t)ctx->stream,
                               (uint64_t)ctx->profiling, (uint64_t)ctx->prof_mask, (uint64_t)ctx->newton_cluster,
                               (uint64_t)ctx->l0_beside});
    }
    if (graphable && ctx->graph_exec && key == ctx->graph_key) {
        LDGA_CUDA(ctx, cudaGraphLaunch(ctx->graph_exec, ctx->stream));
        ctx->n_launches += ctx->graph_launches;
        *replayed_out = true;
        return LDGA_OK;
    }
    TRY(chain_m_enqueue(ctx, a));   // the uncaptured run computes this call's results
    if (graphable) {
        if (ctx->graph_exec) { cudaGraphExecDestroy(ctx->graph_exec); ctx->graph_exec = nullptr; }
        if (ctx->graph) { cudaGraphDestroy(ctx->graph); ctx->graph = nullptr; }
        for (auto& pr : ctx->graph_ev) ctx->ev_free.push_back(pr.second);
        ctx->graph_ev.clear();
        ctx->capturing = true;
        const int64_t n0 = ctx->n_launches;
        cudaError_t e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
        int st = e == cudaSuccess ? chain_m_enqueue(ctx, a) : LDGA_ERR_CUDA;
        cudaGraph_t gr = nullptr;
        cudaError_t e2 = cudaStreamEndCapture(ctx->stream, &gr);
        ctx->capturing = false;
        ctx->graph_launches = ctx->n_launches - n0;   // kernels in the graph (nothing ran yet)
        ctx->n_launches = n0;
        if (e != cudaSuccess || st != LDGA_OK || e2 != cudaSuccess || !gr) {
            if (gr) cudaGraphDestroy(gr);
            cudaGetLastError();
            return ctx_fail(ctx, LDGA_ERR_CUDA, std::string("CUDA graph capture of the chain failed: ") +
                                                    cudaGetErrorString(e != cudaSuccess ? e : e2));
        }
        LDGA_CUDA(ctx, cudaGraphInstantiate(&ctx->graph_exec, gr, 0));
        ctx->graph = gr;
        ctx->graph_key = key;
    }
    return LDGA_OK;
}

// Waits for the handle's stream and unpacks the chain's scalars (layout of ldga_chain_m).
int chain_m_collect(ldga_ctx* ctx, bool replayed, double* scalars_out) {
    TRY(sync(ctx));
    if (replayed && ctx->profiling) {
        for (auto& pr : ctx->graph_ev) {
            float t = 0.f;
            LDGA_CUDA(ctx, cudaEventElapsedTime(&t, ctx->ev_pool[pr.second].a, ctx->ev_pool[pr.second].b));
            ctx->stage_ms[pr.first] += t;
            ctx->stage_cnt[pr.first] += 1;
        }
    }
    const double* r = ctx->h_stage;
    int32_t fails = 0;
    std::memcpy(&fails, reinterpret_cast<const char*>(ctx->h_stage + 64) + sizeof(int32_t), sizeof(int32_t));
    ctx->have_ghat = ctx->have_chi0 = ctx->have_F = ctx->have_lambda0 = ctx->have_sigma = true;
    ctx->have_Gamma[0] = ctx->have_Gamma[1] = ctx->have_chi[0] = ctx->have_chi[1] = true;
    ctx->have_gam[0] = ctx->have_gam[1] = true;
    ctx->sigma_numax = ctx->Nnu / 2;
    if (scalars_out) {
        const double xm = r[8], xd = r[56], U = ctx->mp.U, nn = ctx->mp.n;
        scalars_out[0] = r[16];                                     // λm
        scalars_out[1] = r[24];                                     // μ
        scalars_out[2] = r[25];                                     // E_kin
        scalars_out[3] = r[26];                                     // E_pot,1
        scalars_out[4] = (U / 2.0) * (xd - xm) + U * (nn / 2.0 * nn / 2.0);   // E_pot,2
        scalars_out[5] = (xd + xm) / 2.0;                           // PP_p2 (lhs of the sum rule)
        scalars_out[6] = r[17];                                     // Newton iterations
        scalars_out[7] = r[27];                                     // filling n at μ
    }
    if (fails > 0) return ctx_fail(ctx, LDGA_ERR_NUMERIC, std::to_string(fails) + " BSE matrices are singular or non-finite");
    return LDGA_OK;
}

}  // namespace

int ldga_chain_m(ldga_ctx* ctx, const double* sigma_loc, int32_t n_sigma, const double* gamma_m,
                 const double* gamma_d, const double* chi_loc_m, const double* gimp, int32_t n_gimp,
                 double imp_density, double chiloc_m_sum, int32_t use_graph, double* sigma_out,
                 double* chi_m_out, double* chi_d_out, double* scalars_out) {
    if (!ctx) return ctx_fail(ctx, LDGA_ERR_ARG, "null argument");
    TRY(require_unsharded(ctx, "ldga_chain_m"));
    DeviceGuard g(ctx->device);
    ChainArgs a{sigma_loc, gamma_m, gamma_d, chi_loc_m, gimp, n_sigma, n_gimp, imp_density, chiloc_m_sum,
                sigma_out, chi_m_out, chi_d_out};
    bool replayed = false;
    TRY(chain_m_submit(ctx, a, use_graph != 0, &replayed));
    return chain_m_collect(ctx, replayed, scalars_out);
}

int ldga_batch_chain_m(int32_t n, ldga_ctx* const* ctxs, const ldga_chain_io* io, int32_t use_graph,
                       int32_t* status) {
    if (n < 0 || (n > 0 && (!ctxs || !io))) return ctx_fail(nullptr, LDGA_ERR_ARG, "null argument");
    std::vector<int> st(n, LDGA_OK);
    std::vector<char> rep(n, 0);
    for (int i = 0; i < n; ++i)
        if (ctxs[i] && sharded(ctxs[i])) return require_unsharded(ctxs[i], "ldga_batch_chain_m");
    // every point's chain is in flight before the first wait.  The largest boxes go first: their input
    // copies lead the copy engine's queue and their long BSE launches start while the small points'
    // copies and chains fill in behind them (the order of submission changes no result)
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    auto work = [&](int i) { return ctxs[i] ? (double)ctxs[i]->Nnu * ctxs[i]->Nnu * ctxs[i]->Nw : 0.0; };
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return work(x) > work(y); });
    for (int i : order) {
        ldga_ctx* c = ctxs[i];
        if (!c) { st[i] = LDGA_ERR_ARG; continue; }
        DeviceGuard g(c->device);
        const ldga_chain_io& x = io[i];
        ChainArgs a{x.sigma_loc, x.gamma_m, x.gamma_d, x.chi_loc_m, x.gimp, x.n_sigma, x.n_gimp, x.imp_density,
                    x.chiloc_m_sum, x.sigma_out, x.chi_m_out, x.chi_d_out};
        bool r = false;
        c->l0_beside = n == 1;   // λ₀ beside the BSE only for a chain alone on the GPU
        st[i] = chain_m_submit(c, a, use_graph != 0, &r);
        c->l0_beside = true;
        rep[i] = r;
    }
    int first = LDGA_OK;
    for (int i = 0; i < n; ++i) {
        if (st[i] == LDGA_OK) {
            DeviceGuard g(ctxs[i]->device);
            st[i] = chain_m_collect(ctxs[i], rep[i] != 0, io[i].scalars_out);
        } else if (ctxs[i]) {
            DeviceGuard g(ctxs[i]->device);
            cudaStreamSynchronize(ctxs[i]->stream);   // whatever was enqueued before the failure
        }
        if (status) status[i] = st[i];
        if (first == LDGA_OK && st[i] != LDGA_OK) first = st[i];
    }
    if (first != LDGA_OK) g_create_error = "ldga_batch_chain_m: see status[] and ldga_last_error of each handle";
    return first;
}

// ------------------------------------------------------------------------------- lambda_dm --
namespace {

struct DmState {
    ldga_ctx* ctx;
    double chiloc_m_sum;
    int numax;
    int fix_n = 1;
    double mu;
    double rhs_c1;
    int evals = 0;
    int status = LDGA_OK;
    double last[7];
};

// One residual's device scalars: [0..3] μ, E_kin, E_pot,1, filling (k_mu_fit_energy), [8] sum_kω(χm^λm)
// (the EoM tail's), [9] sum_kω(χd^λd).  Slot k of the three a Newton iteration evaluates.
double* dm_slot(ldga_ctx* ctx, int k) { return ctx->d_red + 128 + 2 * (size_t)ctx->Nnu * ctx->Nw + k * kDmSlot; }

// The residual from a slot's scalars (read back to the host); records μ and the last values in s.
void dm_finish(DmState& s, const double r[kDmSlot], double F[2]) {
    ldga_ctx* ctx = s.ctx;
    const double mu = r[0], ek = r[1], ep1 = r[2], n = r[3], xm = r[8], xd = r[9];
    s.mu = mu;
    const double lhs = (xd + xm) / 2.0;
    const double U = ctx->mp.U, nn = ctx->mp.n;
    const double ep2 = (U / 2.0) * (xd - xm) + U * (nn / 2.0 * nn / 2.0);
    F[0] = lhs - s.rhs_c1;
    F[1] = ep1 - ep2;
    s.last[0] = n; s.last[1] = mu; s.last[2] = ek; s.last[3] = ep1; s.last[4] = ep2; s.last[5] = s.rhs_c1;
    s.last[6] = lhs;
}

// Streams, events and buffers of the residual lanes 1 and 2, made on first use (outside any capture:
// the λdm entry points are not captured).  Lane buffers match the handle's own.
int dm_lanes_ready(ldga_ctx* ctx) {
    if (ctx->dm_stream[0]) return LDGA_OK;
    for (cudaStream_t& st : ctx->dm_stream) LDGA_CUDA(ctx, cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    for (cudaEvent_t* e : {&ctx->dm_ev[0], &ctx->dm_ev[1], &ctx->dm_ev[2], &ctx->dm_fork})
        LDGA_CUDA(ctx, cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    const size_t nsig = (size_t)ctx->Nq * std::max(ctx->Nnu, 1);
    for (int j = 0; j < 2; ++j) {
        LDGA_CUDA(ctx, cudaMalloc(reinterpret_cast<void**>(&ctx->dm_sigma[j]), nsig * sizeof(double2)));
        if (ctx->partial_elems) {
            LDGA_CUDA(ctx, cudaMalloc(reinterpret_cast<void**>(&ctx->dm_partial[j]), ctx->partial_elems * sizeof(double2)));
            ctx->dm_partial_elems[j] = ctx->partial_elems;
        }
    }
    return LDGA_OK;
}

// Lane k's stream, Σ and partial-sum buffers put into the handle (lane 0: the handle's own) by
// lane_enter, and the handle's put back by lane_leave (keeping a lane buffer the EoM may have grown).
struct LaneSave {
    cudaStream_t stream;
    double2 *sigma, *partial;
    size_t partial_elems;
};

void lane_enter(ldga_ctx* ctx, int k, LaneSave& sv) {
    sv = {ctx->stream, ctx->d_sigma, ctx->d_partial, ctx->partial_elems};
    if (k == 0) return;
    const int j = k - 1;
    ctx->stream = ctx->dm_stream[j];
    ctx->d_sigma = ctx->dm_sigma[j];
    ctx->d_partial = ctx->dm_partial[j];
    ctx->partial_elems = ctx->dm_partial_elems[j];
}

void lane_leave(ldga_ctx* ctx, int k, const LaneSave& sv) {
    if (k == 0) return;
    const int j = k - 1;
    ctx->dm_partial[j] = ctx->d_partial;
    ctx->dm_partial_elems[j] = ctx->partial_elems;
    ctx->stream = sv.stream;
    ctx->d_sigma = sv.sigma;
    ctx->d_partial = sv.partial;
    ctx->partial_elems = sv.partial_elems;
}

// residual_vals (conditions_new.jl:250-270) at (lm, ld) into slot k on the current stream: the two χ
// sums in one launch, the EoM, then the μ fit and energies after event `after` (if given), from the
// μ at mu_dev (the previous residual's, on the device) or s.mu
int dm_enqueue(DmState& s, double lm, double ld, int k, cudaEvent_t after, const double* mu_dev) {
    ldga_ctx* ctx = s.ctx;
    double* r = dm_slot(ctx, k);
    TRY(launch_sum_kw2(ctx, lm, ld, r + 8, r + 9));
    TRY(eom_device(ctx, lm, ld, s.numax, 1, s.chiloc_m_sum, r + 8));
    if (after) LDGA_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, after, 0));
    return launch_g_ladder(ctx, s.numax, s.fix_n, s.mu, r, mu_dev);
}

// Residuals at n points (n <= 3) in order, with one host synchronisation.  Residual k runs on lane k:
// its χ sums and EoM overlap the other lanes' work, and its μ fit waits for the μ fit of the residual
// evaluated before it and starts from that μ, as when they run one by one, so the values are the
// same.  A point above 1e5 is not evaluated (NaN residual), as in the reference's residual_vals
// guard.  False on a CUDA or argument error (s.status).
bool dm_residuals(DmState& s, int n, const double (*pts)[2], double (*F)[2]) {
    ldga_ctx* ctx = s.ctx;
    bool eval[3] = {false, false, false};
    const double* mu_src = nullptr;
    int st = n > 1 ? dm_lanes_ready(ctx) : LDGA_OK, last = -1;
    if (!st && n > 1) {
        if (cudaEventRecord(ctx->dm_fork, ctx->stream) != cudaSuccess) st = ctx_fail(ctx, LDGA_ERR_CUDA, "cudaEventRecord");
        for (int j = 0; j < 2 && !st; ++j)
            if (cudaStreamWaitEvent(ctx->dm_stream[j], ctx->dm_fork, 0) != cudaSuccess)
                st = ctx_fail(ctx, LDGA_ERR_CUDA, "cudaStreamWaitEvent");
    }
    for (int k = 0; k < n && !st; ++k) {
        s.evals++;
        if (pts[k][0] > 1e5 || pts[k][1] > 1e5) continue;
        LaneSave sv;
        lane_enter(ctx, k, sv);
        st = dm_enqueue(s, pts[k][0], pts[k][1], k, last >= 0 ? ctx->dm_ev[last] : nullptr, mu_src);
        if (!st && n > 1 && cudaEventRecord(ctx->dm_ev[k], ctx->stream) != cudaSuccess)
            st = ctx_fail(ctx, LDGA_ERR_CUDA, "cudaEventRecord");
        lane_leave(ctx, k, sv);
        eval[k] = true;
        mu_src = dm_slot(ctx, k);
        last = k;
    }
    for (int k = 1; k < n && !st; ++k)   // join the lanes before the read-back
        if (eval[k] && cudaStreamWaitEvent(ctx->stream, ctx->dm_ev[k], 0) != cudaSuccess)
            st = ctx_fail(ctx, LDGA_ERR_CUDA, "cudaStreamWaitEvent");
    double r[3][kDmSlot];
    if (!st && last >= 0) st = copy(ctx, r, dm_slot(ctx, 0), (size_t)(last + 1) * kDmSlot * sizeof(double));
    if (!st && last >= 0) st = sync(ctx);
    if (st) {
        if (n > 1)   // nothing of this call stays in flight on the lanes
            for (cudaStream_t ls : ctx->dm_stream)
                if (ls) cudaStreamSynchronize(ls);
        s.status = st;
        return false;
    }
    for (int k = 0; k < n; ++k) {
        if (eval[k]) dm_finish(s, r[k], F[k]);
        else F[k][0] = F[k][1] = NAN;
    }
    return true;
}

bool dm_residual(DmState& s, double lm, double ld, double F[2]) {
    const double p[1][2] = {{lm, ld}};
    double f[1][2];
    if (!dm_residuals(s, 1, p, f)) return false;
    F[0] = f[0][0];
    F[1] = f[0][1];
    return true;
}

double fd_step(double x) {
    const double r = std::sqrt(2.220446049250313e-16);
    return std::max(r * std::fabs(x), r);
}

// newton_right, N-D (LambdaCorrection/helpers.jl:165-208) on the λdm residual; false on a CUDA or
// argument error (s.status), *failed when the back-off resets are exhausted.
bool dm_newton(DmState& s, const double start[2], const double xmin[2], double atol, int nsteps, double xi[2],
               int* iters, bool* failed_out) {
    xi[0] = start[0]; xi[1] = start[1];
    int i = 1, reset_i = 1;
    bool bis_fail = false, failed = false;
    const int max_reset = 5;
    const double reset_backoff = 1.0;
    while (true) {
        double fi[2], J[2][2];
        // f at xi and the forward-difference Jacobian's two points, enqueued together (one host
        // synchronisation).  FiniteDiff evaluates f(x) once more; the residual is a deterministic
        // function of x (its μ fit converges to |Δn| < 1e-14 from any warm start), so the value
        // at xi is used
        const double e[2] = {fd_step(xi[0]), fd_step(xi[1])};
        const double pts[3][2] = {{xi[0], xi[1]}, {xi[0] + e[0], xi[1]}, {xi[0], xi[1] + e[1]}};
        double f3[3][2];
        if (s.ctx->dm_lanes) {
            if (!dm_residuals(s, 3, pts, f3)) return false;
        } else {
            for (int k = 0; k < 3; ++k)
                if (!dm_residuals(s, 1, pts + k, f3 + k)) return false;
        }
        fi[0] = f3[0][0];
        fi[1] = f3[0][1];
        for (int j = 0; j < 2; ++j) {
            J[0][j] = (f3[1 + j][0] - fi[0]) / e[j];
            J[1][j] = (f3[1 + j][1] - fi[1]) / e[j];
        }
        const double det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
        const double inv[2][2] = {{J[1][1] / det, -J[0][1] / det}, {-J[1][0] / det, J[0][0] / det}};
        const double last[2] = {xi[0], xi[1]};
        xi[0] = xi[0] - (inv[0][0] * fi[0] + inv[0][1] * fi[1]);
        xi[1] = xi[1] - (inv[1][0] * fi[0] + inv[1][1] * fi[1]);
        for (int l = 0; l < 2; ++l) {
            if (xi[l] < xmin[l]) {
                xi[l] = xmin[l] + std::fabs(last[l] - xmin[l]) / 2.0;
                if (std::fabs(last[l] - xmin[l]) / 2.0 < 1e-8) bis_fail = true;
            }
        }
        if (bis_fail || !std::isfinite(fi[0]) || !std::isfinite(fi[1])) {
            bis_fail = false;
            if (reset_i >= max_reset) { failed = true; break; }
            reset_i += 1;
            xi[0] = start[0] + reset_i * reset_backoff * std::fabs(xmin[0]);
            xi[1] = start[1] + reset_i * reset_backoff * std::fabs(xmin[1]);
        }
        if (std::fabs(std::sqrt(fi[0] * fi[0] + fi[1] * fi[1])) < atol) break;
        if (i >= nsteps) break;
        i += 1;
    }
    *iters = i;
    *failed_out = failed;
    return true;
}

}  // namespace

int ldga_lambda_dm(ldga_ctx* ctx, double chiloc_m_sum, int32_t numax, double lam_min_delta, double atol,
                   int32_t nsteps, double* lam_m, double* lam_d, int32_t* converged, double* out7,
                   int32_t* numax_out, double* sigma_out, double* G_out) {
    if (!ctx || !lam_m || !lam_d) return ctx_fail(ctx, LDGA_ERR_ARG, "null argument");
    TRY(require_unsharded(ctx, "ldga_lambda_dm"));
    TRY(eom_inputs_ready(ctx));
    NEED(ctx, ctx->d_sigma_loc != nullptr, "λdm_correction: Sigma_loc missing (call ldga_gloc)");
    DeviceGuard g(ctx->device);
    const int nw_use = ctx->Nw;   // usable range = full range (chi built with full_range = true)
    int nu_auto = std::min(ctx->sp.n_iv, (int)std::floor(3.0 * nw_use / 8.0));
    if (ctx->sp.dbg_full_eom_omega) nu_auto = std::min(ctx->sp.n_iv, (int)std::floor(3.0 * ctx->Nw / 8.0));
    const int nu = numax < 1 ? nu_auto : std::min(nu_auto, (int)numax);
    if (nu < 1) return ctx_fail(ctx, LDGA_ERR_ARG, "λdm: no fermionic frequencies for the EoM");
    if (numax_out) *numax_out = nu;
    DmState s;
    s.ctx = ctx; s.chiloc_m_sum = chiloc_m_sum; s.numax = nu; s.mu = ctx->mp.mu;
    s.rhs_c1 = ctx->mp.n / 2.0 * (1.0 - ctx->mp.n / 2.0);
    // bounds: lambda_min + delta |lambda_min| (conditions_new.jl:290-293)
    double lmin[2];
    TRY(launch_lambda_min(ctx, LDGA_CH_M, ctx->d_red + 40));
    TRY(launch_lambda_min(ctx, LDGA_CH_D, ctx->d_red + 41));
    TRY(copy(ctx, lmin, ctx->d_red + 40, 2 * sizeof(double)));
    TRY(sync(ctx));
    const double xmin[2] = {lmin[0] + lam_min_delta * std::fabs(lmin[0]), lmin[1] + lam_min_delta * std::fabs(lmin[1])};
    const double start[2] = {0.0, 0.0};
    double xi[2];
    int i = 0;
    bool failed = false;
    if (!dm_newton(s, start, xmin, atol, nsteps, xi, &i, &failed)) return s.status;
    ctx->lambda_dm_evals = s.evals;
    if (failed || !std::isfinite(xi[0]) || !std::isfinite(xi[1])) {
        *lam_m = NAN; *lam_d = NAN;
        if (converged) *converged = 0;
        if (out7) for (int k = 0; k < 7; ++k) out7[k] = NAN;
        return ctx_fail(ctx, LDGA_ERR_NOCONV, "λ root-finding failed after " + std::to_string(i) + " iterations");
    }
    double F[2];
    if (!dm_residual(s, xi[0], xi[1], F)) return s.status;
    ctx->lambda_dm_evals = s.evals;
    *lam_m = xi[0];
    *lam_d = xi[1];
    const bool conv = std::fabs(s.rhs_c1 - s.last[6]) <= 1e-8 && std::fabs(s.last[3] - s.last[4]) <= 1e-8;
    if (converged) *converged = conv ? 1 : 0;
    if (out7) for (int k = 0; k < 7; ++k) out7[k] = s.last[k];
    if (sigma_out) TRY(copy(ctx, sigma_out, ctx->d_sigma, (size_t)ctx->Nq * nu * sizeof(double2)));
    if (G_out) {
        TRY(launch_g_ladder_full(ctx, nu, ctx->d_red + 24));
        TRY(copy(ctx, G_out, ctx->d_gladder, (size_t)ctx->Nq * ctx->Nf * sizeof(double2)));
    }
    return sync(ctx);
}

// ------------------------------------------------------------------------------- run_sc ----
namespace {
// Sigma <- (1 - a) Sigma + a Sigma_old  (run_sc!, conditions_new.jl:469)
__global__ void k_sigma_mix(double2* sigma, const double2* old, size_t n, double a) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const double2 x = sigma[e], y = old[e];
        sigma[e] = make_double2((1.0 - a) * x.x + a * y.x, (1.0 - a) * x.y + a * y.y);
    }
}

// Device buffers of one run_sc call, freed on every exit path.
struct ScBuffers {
    double2 *sigma_old = nullptr, *ghat_save = nullptr, *gloc_save = nullptr;
    double* chi_save = nullptr;   // update_χ_tail: both channels' chi, restored on return
    ~ScBuffers() {
        if (sigma_old) cudaFree(sigma_old);
        if (ghat_save) cudaFree(ghat_save);
        if (gloc_save) cudaFree(gloc_save);
        if (chi_save) cudaFree(chi_save);
    }
};

// The χ tail update of run_sc! changes the handle's chi data and the c2 tail coefficient (ModelParameters'
// E_kin_DMFT, which the sums use); both are put back when the loop returns, also on errors.
struct TailRestore {
    ldga_ctx* ctx = nullptr;
    double* chi_save = nullptr;
    double ekin = 0.0;
    ~TailRestore() {
        if (!ctx) return;
        const size_t n = (size_t)ctx->Nq * ctx->Nw;
        cudaMemcpyAsync(ctx->d_chi[0], chi_save, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream);
        cudaMemcpyAsync(ctx->d_chi[1], chi_save + n, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream);
        cudaStreamSynchronize(ctx->stream);
        ctx->mp.Ekin_DMFT = ekin;
    }
};
}  // namespace

int ldga_run_sc(ldga_ctx* ctx, double lam_m, double lam_d, int32_t flags, double mu, double chiloc_m_sum,
                int32_t numax, int32_t maxit, double mixing, double conv_abs, int32_t fit_mu, double lam_min_delta,
                double* out, double* sigma_out, double* G_out) {
    if (!ctx || !out) return ctx_fail(ctx, LDGA_ERR_ARG, "null argument");
    TRY(require_unsharded(ctx, "ldga_run_sc"));
    const bool redo_dm = (flags & LDGA_SC_REDO_DM) != 0;
    const bool update_tail = (flags & LDGA_SC_UPDATE_CHI_TAIL) != 0;
    const bool lam_types = (flags & LDGA_SC_LAMBDA_TYPE) != 0;
    TRY(eom_inputs_ready(ctx));
    NEED(ctx, ctx->d_sigma_loc != nullptr, "run_sc: Sigma_loc missing (call ldga_gloc)");
    NEED(ctx, ctx->have_ghat, "run_sc: G missing (call ldga_gloc or ldga_set_gloc)");
    if (!std::isfinite(lam_m) || !std::isfinite(lam_d)) return ctx_fail(ctx, LDGA_ERR_ARG, "λ must be finite");
    if (maxit < 1) return ctx_fail(ctx, LDGA_ERR_ARG, "maxit must be >= 1");
    DeviceGuard g(ctx->device);
    int nu = std::min(ctx->sp.n_iv, (int)std::floor(3.0 * ctx->Nw / 8.0));   // gen_νω_indices νGrid
    if (numax >= 1) nu = std::min(nu, (int)numax);
    if (nu < 1) return ctx_fail(ctx, LDGA_ERR_ARG, "run_sc: no fermionic frequencies for the EoM");
    const size_t nsig = (size_t)ctx->Nq * nu, ngf = (size_t)ctx->Nq * ctx->Nf;
    ScBuffers b;
    TRY(dev_alloc(ctx, &b.sigma_old, nsig));
    TRY(dev_alloc(ctx, &b.ghat_save, ngf));
    TRY(dev_alloc(ctx, &b.gloc_save, ngf));
    // the reference works on deepcopy(h.gLoc_rfft): the handle's G and its transform are restored at the end
    TRY(copy(ctx, b.ghat_save, ctx->d_ghat, ngf * sizeof(double2)));
    TRY(copy(ctx, b.gloc_save, ctx->d_gloc, ngf * sizeof(double2)));
    LDGA_CUDA(ctx, cudaMemsetAsync(ctx->d_sigma, 0, nsig * sizeof(double2), ctx->stream));

    const double U = ctx->mp.U, nn = ctx->mp.n;
    const double rhs_c1 = nn / 2.0 * (1.0 - nn / 2.0);
    double lm = lam_m, ld = lam_d;
    auto sums = [&](double* lhs, double* ep2) -> int {
        double r[2];
        TRY(launch_sum_kw2(ctx, lm, ld, ctx->d_red + 32, ctx->d_red + 33));
        TRY(copy(ctx, r, ctx->d_red + 32, 2 * sizeof(double)));
        TRY(sync(ctx));
        *lhs = (r[1] + r[0]) / 2.0;
        *ep2 = (U / 2.0) * (r[1] - r[0]) + U * (nn / 2.0 * nn / 2.0);
        return LDGA_OK;
    };
    TailRestore restore;
    if (update_tail) {
        const size_t nqw = (size_t)ctx->Nq * ctx->Nw;
        TRY(dev_alloc(ctx, &b.chi_save, 2 * nqw));
        TRY(copy(ctx, b.chi_save, ctx->d_chi[0], nqw * sizeof(double)));
        TRY(copy(ctx, b.chi_save + nqw, ctx->d_chi[1], nqw * sizeof(double)));
        restore.ctx = ctx;
        restore.chi_save = b.chi_save;
        restore.ekin = ctx->mp.Ekin_DMFT;
    }
    double lhs_c1 = 0.0, E_pot_2 = 0.0, E_pot_1 = INFINITY, E_kin = INFINITY, n_fill = NAN;
    TRY(sums(&lhs_c1, &E_pot_2));
    bool converged = false;
    int it = 1, iters = 0, tail_it = 1;
    double r[4] = {mu, NAN, NAN, NAN};
    for (;;) {   // χ tail updates (one pass without update_χ_tail)
    while (true) {
        if (it > 1 && redo_dm) {
            // λdm_correction on the current G transform, from the previous root (conditions_new.jl:431-436)
            DmState s;
            s.ctx = ctx; s.chiloc_m_sum = chiloc_m_sum; s.numax = nu; s.mu = mu; s.fix_n = fit_mu ? 1 : 0;
            s.rhs_c1 = rhs_c1;
            double lmin[2];
            TRY(launch_lambda_min(ctx, LDGA_CH_M, ctx->d_red + 40));
            TRY(launch_lambda_min(ctx, LDGA_CH_D, ctx->d_red + 41));
            TRY(copy(ctx, lmin, ctx->d_red + 40, 2 * sizeof(double)));
            TRY(sync(ctx));
            const double xmin[2] = {lmin[0] + lam_min_delta * std::fabs(lmin[0]), lmin[1] + lam_min_delta * std::fabs(lmin[1])};
            const double start[2] = {lm, ld};
            double xi[2];
            int ni = 0;
            bool failed = false;
            if (!dm_newton(s, start, xmin, 1e-8, 500, xi, &ni, &failed)) return s.status;
            // a failed root ends the loop with NaN λ and μ; a found one always counts as valid there
            // (the inner λ_result's `converged` field is true for every root, conditions_new.jl:314)
            if (failed || !std::isfinite(xi[0]) || !std::isfinite(xi[1])) { lm = NAN; ld = NAN; mu = NAN; break; }
            double F[2];
            if (!dm_residual(s, xi[0], xi[1], F)) return s.status;
            lm = xi[0]; ld = xi[1]; mu = s.mu;
        }
        TRY(copy(ctx, b.sigma_old, ctx->d_sigma, nsig * sizeof(double2)));
        TRY(eom_device(ctx, lm, ld, nu, 1, chiloc_m_sum));
        if (mixing != 0.0 && it > 1) {
            k_sigma_mix<<<2 * 148, 256, 0, ctx->stream>>>(ctx->d_sigma, b.sigma_old, nsig, mixing);
            LDGA_LAUNCHED(ctx, "k_sigma_mix");
        }
        // G_from_Σladder! (μ fit), calc_E, filling_pos, then the G transform for the next EoM
        TRY(launch_g_ladder(ctx, nu, fit_mu ? 1 : 0, mu, ctx->d_red + 24));
        TRY(launch_g_ladder_full(ctx, nu, ctx->d_red + 24));
        TRY(copy(ctx, r, ctx->d_red + 24, 4 * sizeof(double)));
        TRY(sync(ctx));
        iters = it;
        if (std::isnan(r[0])) break;
        mu = r[0];
        const double E_pot_1_old = E_pot_1, E_pot_2_old = E_pot_2;
        E_kin = r[1]; E_pot_1 = r[2]; n_fill = r[3];
        TRY(copy(ctx, ctx->d_gloc, ctx->d_gladder, ngf * sizeof(double2)));
        TRY(launch_gloc_transform(ctx, false));
        TRY(sums(&lhs_c1, &E_pot_2));
        if (std::fabs(E_pot_1 - E_pot_1_old) < conv_abs && std::fabs(E_pot_2 - E_pot_2_old) < conv_abs) {
            converged = true;
            break;
        }
        if (it >= maxit) break;
        it += 1;
    }
    if (!update_tail) break;
    // conditions_new.jl:519-545: c2 = E_kin on both channels (update_tail!), the sum rules again, and
    // a restarted loop (it = 1) unless they hold or 20 updates were made
    if (!std::isfinite(E_kin)) {
        E_pot_1 = NAN;
    } else {
        const double dc2 = E_kin - ctx->mp.Ekin_DMFT;
        if (dc2 != 0.0) {
            TRY(launch_chi_tail_shift(ctx, LDGA_CH_M, dc2));
            TRY(launch_chi_tail_shift(ctx, LDGA_CH_D, dc2));
            ctx->mp.Ekin_DMFT = E_kin;
        }
    }
    TRY(sums(&lhs_c1, &E_pot_2));
    if (tail_it >= 20 || (std::fabs(E_pot_1 - E_pot_2) < conv_abs && std::fabs(lhs_c1 - rhs_c1) < conv_abs)) break;
    it = 1;
    if (lam_types) { lm = 0.0; ld = 0.0; }   // run_sc! takes the first λ of a loop from χ.λ, 0 after a pass
    tail_it += 1;
    }
    if (sigma_out) TRY(copy(ctx, sigma_out, ctx->d_sigma, nsig * sizeof(double2)));
    if (G_out) TRY(copy(ctx, G_out, ctx->d_gladder, ngf * sizeof(double2)));
    TRY(copy(ctx, ctx->d_ghat, b.ghat_save, ngf * sizeof(double2)));
    TRY(copy(ctx, ctx->d_gloc, b.gloc_save, ngf * sizeof(double2)));
    TRY(sync(ctx));
    ctx->sigma_numax = nu;
    // out: λm, λd, rhs_c1, lhs_c1, E_pot_1, E_pot_2, E_kin, n, μ, sc_converged, iterations, νmax
    const double vals[12] = {lm, ld, rhs_c1, lhs_c1, E_pot_1, E_pot_2, E_kin, n_fill, mu, converged ? 1.0 : 0.0,
                             (double)iters, (double)nu};
    for (int k = 0; k < 12; ++k) out[k] = vals[k];
    return LDGA_OK;
}

int ldga_lambda_dm_evals(const ldga_ctx* ctx, int32_t* n_evals) {
    if (!ctx || !n_evals) return LDGA_ERR_ARG;
    *n_evals = ctx->lambda_dm_evals;
    return LDGA_OK;
}

}  // extern "C"
