// a7: batched Bethe-Salpeter solve (calc_χγ, BSETools.jl:192-248; inv! LapackWrapper.jl:64-72).
//
// For every (q, w) the reference inverts A = Gamma_r(w) + diag(1/chi0(q, :, w)) with zgetrf+zgetri
// and only uses y = (1^T A^-1)^T, i.e. the solution of B y = 1 with B = A^T:
//     chi_r(q, w) = Re(sum_nu y_nu) / beta^2,   gamma_r(q, nu, w) = y_nu / (chi0(q,nu,w)(1 + s U chi_r)).
//
// Kernel layout: one CTA per (w, chunk of q); Gamma(w) is staged once in shared memory (FP64) and
// reused by every q of the chunk.  Row i of B lives in the registers of H adjacent lanes (lane h
// of the group holds the columns j = s*H + h), so a Gauss-Jordan step k is: the owners of row k
// publish it to shared memory (double-buffered, one barrier per step), every other row computes
// its multiplier m = b_ik / b_kk in the lane that owns column k, broadcasts it within the group by
// shuffle, and updates its remaining columns.  All loops are unrolled at compile time, so every
// register index is static and the column bound j > k costs no predicated work outside one slot.
//
// Modes:
//   LDGA_PREC_FP64_INV  in-place FP64 Gauss-Jordan inverse (N^3, the reference's formulation);
//                       y = row sums of B^-1.
//   LDGA_PREC_FP64      FP64 Gauss-Jordan elimination of [B | 1] (N^3/2).
//   LDGA_PREC_MIXED     FP32 elimination with the multipliers kept, then FP64 iterative refinement:
//                       r = 1 - B y in FP64 (Gamma from shared memory), delta from the stored FP32
//                       elimination, y += delta, until the update is below FP64 resolution.
// No pivoting is done in the fast path.  Every solution is verified by its FP64 backward error
// |1 - B y|_inf / (|B|_inf |y|_inf + 1); a matrix above 1e-12 (or with a non-finite y) is flagged
// and re-solved by a partial-pivoting FP64 LU kernel, which is also the path for box sizes that
// have no unrolled instantiation.
#include <cmath>
#include <cstdio>

#include "ldga_internal.cuh"

namespace {

template <typename TF> struct C2;
template <> struct C2<double> { using T = double2; };
template <> struct C2<float> { using T = float2; };

template <typename V>
__device__ __forceinline__ V vmk(double r, double i) { V v; v.x = r; v.y = i; return v; }

template <typename V>
__device__ __forceinline__ V vmul(V a, V b) {
    V r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
// a -= m * b
template <typename V>
__device__ __forceinline__ void vfnms(V& a, V m, V b) {
    a.x = fma(-m.x, b.x, a.x);
    a.x = fma(m.y, b.y, a.x);
    a.y = fma(-m.x, b.y, a.y);
    a.y = fma(-m.y, b.x, a.y);
}
template <typename V>
__device__ __forceinline__ V vinv(V z) {
    using R = decltype(z.x);
    R s = fabs(z.x) > fabs(z.y) ? fabs(z.x) : fabs(z.y);
    R xr = z.x / s, xi = z.y / s;
    R d = (xr * xr + xi * xi) * s;
    V r; r.x = xr / d; r.y = -xi / d; return r;
}

template <typename V>
__device__ __forceinline__ V shfl_v(V v, int src, int width) {
    V r;
    r.x = __shfl_sync(0xffffffffu, v.x, src, width);
    r.y = __shfl_sync(0xffffffffu, v.y, src, width);
    return r;
}

struct BseArgs {
    int nq, nnu, nw, qchunk;
    double beta, U;
    int s;            // -1 for d, +1 for m
    const double2* Gamma;   // [Nnu, Nnu, Nw]
    const double2* chi0;    // [Nq, Nnu, Nw]
    double* chi;            // [Nq, Nw]
    double2* gam;           // [Nq, Nnu, Nw]
    int32_t* flags;         // [Nq, Nw]
};

__device__ __forceinline__ double2 dmk(double r, double i) { return make_double2(r, i); }

// Block-wide sum in a fixed order (deterministic): lanes -> warps -> warp 0.
__device__ __forceinline__ double block_sum_det(double v, double* red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    double r = 0.0;
    const int nw = (blockDim.x + 31) >> 5;
    for (int i = 0; i < nw; ++i) r += red[i];
    return r;
}
__device__ __forceinline__ double block_max(double v, double* red) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    double r = 0.0;
    const int nw = (blockDim.x + 31) >> 5;
    for (int i = 0; i < nw; ++i) r = fmax(r, red[i]);
    return r;
}

template <int N, int H, typename TF, int MODE>
__global__ void __launch_bounds__(((N * H + 31) / 32) * 32) k_bse_gj(const BseArgs a) {
    using V = typename C2<TF>::T;
    constexpr int S = (N + H - 1) / H;
    extern __shared__ double2 sm[];
    double2* Gsm = sm;                               // [N*N] Gamma(w), Julia layout G[j + N*i]
    V* rowbuf = reinterpret_cast<V*>(Gsm + N * N);   // [2][N + 1] published row k (+ rhs)
    double2* ysm = reinterpret_cast<double2*>(rowbuf + 2 * (N + 1));   // [N]
    double* red = reinterpret_cast<double*>(ysm + N);                 // [32]
    V* zsm = reinterpret_cast<V*>(red + 32);                           // [N] refinement rhs

    const int w = blockIdx.y;
    const int q0 = blockIdx.x * a.qchunk;
    const int q1 = min(a.nq, q0 + a.qchunk);
    const int tid = threadIdx.x;
    const int i = tid / H, h = tid - (tid / H) * H;
    const bool act = i < N;
    const int lane = tid & 31;
    const int gbase = lane - h;      // first lane of this row's group

    const double2* Gw = a.Gamma + (size_t)w * N * N;
    for (int e = tid; e < N * N; e += blockDim.x) Gsm[e] = Gw[e];
    __syncthreads();

    for (int q = q0; q < q1; ++q) {
        // ---- load row i of B = A^T: B_ij = Gamma[j, i] + delta_ij / chi0(q, i, w)
        const size_t ci = act ? ((size_t)q + (size_t)a.nq * (i + (size_t)N * w)) : 0;
        double2 c0 = act ? a.chi0[ci] : dmk(1.0, 0.0);
        double2 dii = cinv(c0);
        V b[S];
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const int j = s * H + h;
            double2 g = (act && j < N) ? Gsm[i * N + j] : dmk(0.0, 0.0);
            if (j == i) g = cadd(g, dii);
            b[s] = vmk<V>(g.x, g.y);
        }
        V z = vmk<V>(1.0, 0.0);
        V mypiv = vmk<V>(1.0, 0.0);

        // ---- elimination
#pragma unroll
        for (int k = 0; k < N; ++k) {
            const int sk = k / H, hk = k - (k / H) * H;
            V* rb = rowbuf + (k & 1) * (N + 1);
            if (act && i == k) {
#pragma unroll
                for (int s = 0; s < S; ++s) {
                    const int j = s * H + h;
                    if (MODE == LDGA_PREC_FP64_INV) {
                        if (j < N) rb[j] = b[s];
                    } else {
                        if (s >= sk && j < N) rb[j] = b[s];
                    }
                }
                if (h == 0) rb[N] = z;
            }
            __syncthreads();
            const V piv = rb[k];
            const V inv = vinv<V>(piv);
            if (i == k) mypiv = piv;
            if (MODE == LDGA_PREC_FP64_INV) {
                // in-place Gauss-Jordan inverse: row k scaled by 1/p (b_kk -> 1/p), others
                // b_ij -= b_ik * row_k[j] / p with b_ik -> -b_ik / p
                V f = vmk<V>(0.0, 0.0);
                if (h == hk) f = b[sk];
                f = shfl_v<V>(f, gbase + hk, 32);
                if (i == k) {
#pragma unroll
                    for (int s = 0; s < S; ++s) {
                        const int j = s * H + h;
                        if (j == k) b[s] = inv; else b[s] = vmul<V>(b[s], inv);
                    }
                } else {
                    if (h == hk) b[sk] = vmk<V>(0.0, 0.0);
#pragma unroll
                    for (int s = 0; s < S; ++s) {
                        const int j = s * H + h;
                        if (j < N) {
                            V u = (j == k) ? inv : vmul<V>(rb[j], inv);
                            vfnms<V>(b[s], f, u);
                        }
                    }
                }
            } else {
                V m = vmk<V>(0.0, 0.0);
                if (h == hk) {
                    m = vmul<V>(b[sk], inv);
                    if (i != k) b[sk] = m;          // keep the multiplier for refinement
                }
                m = shfl_v<V>(m, gbase + hk, 32);
                if (i != k) {
#pragma unroll
                    for (int s = 0; s < S; ++s) {
                        if (s >= sk) {
                            const int j = s * H + h;
                            if (j > k && j < N) vfnms<V>(b[s], m, rb[j]);
                        }
                    }
                    vfnms<V>(z, m, rb[N]);
                }
            }
        }

        // ---- solution y (FP64)
        double2 y = dmk(0.0, 0.0);
        if (MODE == LDGA_PREC_FP64_INV) {
            // y_i = sum_j X_ij
            double2 part = dmk(0.0, 0.0);
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const int j = s * H + h;
                if (j < N) part = cadd(part, dmk((double)b[s].x, (double)b[s].y));
            }
#pragma unroll
            for (int o = 1; o < H; o <<= 1) {
                part.x += __shfl_xor_sync(0xffffffffu, part.x, o, 32);
                part.y += __shfl_xor_sync(0xffffffffu, part.y, o, 32);
            }
            y = part;
        } else {
            const V t = vmul<V>(z, vinv<V>(mypiv));
            y = dmk((double)t.x, (double)t.y);
        }
        if (act && h == 0) ysm[i] = y;
        __syncthreads();

        // ---- FP64 residual r_i = 1 - sum_j B_ij y_j and (MIXED) refinement
        bool ok = true;
        const int max_ref = (MODE == LDGA_PREC_MIXED) ? 6 : 0;
        double bnorm_row = 0.0;
        for (int it = 0; it <= max_ref; ++it) {
            double2 acc = dmk(0.0, 0.0);
            double rown = 0.0;
            if (act) {
#pragma unroll
                for (int s = 0; s < S; ++s) {
                    const int j = s * H + h;
                    if (j < N) {
                        double2 g = Gsm[i * N + j];
                        if (j == i) g = cadd(g, dii);
                        acc = cadd(acc, cmul(g, ysm[j]));
                        rown += fabs(g.x) + fabs(g.y);
                    }
                }
            }
#pragma unroll
            for (int o = 1; o < H; o <<= 1) {
                acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o, 32);
                acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o, 32);
                rown += __shfl_xor_sync(0xffffffffu, rown, o, 32);
            }
            const double2 r = dmk(1.0 - acc.x, -acc.y);
            const double rabs = act ? fabs(r.x) + fabs(r.y) : 0.0;
            const double yabs = act ? fabs(y.x) + fabs(y.y) : 0.0;
            const double rmax = block_max(rabs, red);
            const double ymax = block_max(yabs, red);
            bnorm_row = block_max(act ? rown : 0.0, red);
            const double berr = rmax / (bnorm_row * ymax + 1.0);
            const bool finite = isfinite(berr);
            if (MODE != LDGA_PREC_MIXED || it == max_ref) {
                ok = finite && berr <= 1e-12;
                break;
            }
            if (!finite) { ok = false; break; }
            if (berr <= 2e-16) { ok = true; break; }
            // delta = (stored FP32 elimination) applied to r
            if (act && h == 0) zsm[i] = vmk<V>(r.x, r.y);
            __syncthreads();
#pragma unroll
            for (int k = 0; k < N; ++k) {
                const int sk = k / H, hk = k - (k / H) * H;
                const V zk = zsm[k];
                if (act && i != k && h == hk) {
                    V zi = zsm[i];
                    vfnms<V>(zi, b[sk], zk);
                    zsm[i] = zi;
                }
                __syncthreads();
            }
            if (act && h == 0) {
                const V d = vmul<V>(zsm[i], vinv<V>(mypiv));
                y = cadd(y, dmk((double)d.x, (double)d.y));
                ysm[i] = y;
            }
            // other lanes of the group need the updated y only through ysm
            __syncthreads();
            if (act) y = ysm[i];
        }

        // ---- chi and gamma
        const double ysum = block_sum_det((act && h == 0) ? y.x : 0.0, red);
        const double chi = ysum / (a.beta * a.beta);
        if (tid == 0) {
            a.chi[(size_t)q + (size_t)a.nq * w] = chi;
            a.flags[(size_t)q + (size_t)a.nq * w] = ok ? 0 : 1;
        }
        if (act && h == 0) {
            const double f = 1.0 + a.s * a.U * chi;
            a.gam[ci] = cdiv(y, cscale(c0, f));
        }
        __syncthreads();
    }
}

// Fallback: partial-pivoting FP64 LU of B = A^T (one matrix per CTA, shared memory), used for flagged
// matrices and for box sizes without an unrolled instantiation.  list == nullptr: all (q, w).
__global__ void __launch_bounds__(256) k_bse_lu_pivot(const BseArgs a, const int32_t* list, int count,
                                                       const int32_t* count_dev) {
    extern __shared__ double2 sm[];
    const int N = a.nnu;
    double2* B = sm;                 // [N][N+1] row-major, last column = rhs
    double* red = reinterpret_cast<double*>(B + N * (N + 1));
    int* piv_s = reinterpret_cast<int*>(red + 64);
    const int ld = N + 1;
    if (count_dev) count = count_dev[0];
    for (int item = blockIdx.x; item < count; item += gridDim.x) {
        const int lin = list ? list[item] : item;
        const int q = lin % a.nq, w = lin / a.nq;
        const double2* Gw = a.Gamma + (size_t)w * N * N;
        for (int e = threadIdx.x; e < N * N; e += blockDim.x) {
            const int ii = e / N, j = e - ii * N;
            double2 g = Gw[(size_t)ii * N + j];       // Gamma[j, ii] -> B[ii][j]
            if (ii == j) g = cadd(g, cinv(a.chi0[(size_t)q + (size_t)a.nq * (ii + (size_t)N * w)]));
            B[ii * ld + j] = g;
        }
        for (int ii = threadIdx.x; ii < N; ii += blockDim.x) B[ii * ld + N] = dmk(1.0, 0.0);
        __syncthreads();
        for (int k = 0; k < N; ++k) {
            // pivot search (cabs1, as izamax) by warp 0
            if (threadIdx.x < 32) {
                double best = -1.0;
                int bi = k;
                for (int r = k + threadIdx.x; r < N; r += 32) {
                    const double v = fabs(B[r * ld + k].x) + fabs(B[r * ld + k].y);
                    if (v > best) { best = v; bi = r; }
                }
                for (int o = 16; o > 0; o >>= 1) {
                    const double ob = __shfl_down_sync(0xffffffffu, best, o);
                    const int oi = __shfl_down_sync(0xffffffffu, bi, o);
                    if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
                }
                if (threadIdx.x == 0) piv_s[0] = bi;
            }
            __syncthreads();
            const int p = piv_s[0];
            if (p != k) {
                for (int j = threadIdx.x; j <= N; j += blockDim.x) {
                    const double2 t = B[k * ld + j];
                    B[k * ld + j] = B[p * ld + j];
                    B[p * ld + j] = t;
                }
            }
            __syncthreads();
            const double2 inv = cinv(B[k * ld + k]);
            const int rows = N - k - 1, cols = N - k;   // columns k+1..N (incl. rhs)
            for (int e = threadIdx.x; e < rows * cols; e += blockDim.x) {
                const int r = k + 1 + e / cols, j = k + 1 + e % cols;
                const double2 m = cmul(B[r * ld + k], inv);
                B[r * ld + j] = csub(B[r * ld + j], cmul(m, B[k * ld + j]));
            }
            __syncthreads();
        }
        // back substitution (serial in k, parallel dot products)
        for (int k = N - 1; k >= 0; --k) {
            double2 part = dmk(0.0, 0.0);
            for (int j = k + 1 + threadIdx.x; j < N; j += blockDim.x) part = cadd(part, cmul(B[k * ld + j], B[j * ld + N]));
            double re = block_sum_det(part.x, red);
            double im = block_sum_det(part.y, red);
            if (threadIdx.x == 0) B[k * ld + N] = cdiv(csub(B[k * ld + N], dmk(re, im)), B[k * ld + k]);
            __syncthreads();
        }
        double ys = 0.0;
        for (int ii = threadIdx.x; ii < N; ii += blockDim.x) ys += B[ii * ld + N].x;
        const double chi = block_sum_det(ys, red) / (a.beta * a.beta);
        if (threadIdx.x == 0) {
            a.chi[(size_t)q + (size_t)a.nq * w] = chi;
            a.flags[(size_t)q + (size_t)a.nq * w] = isfinite(chi) ? 0 : 2;
        }
        const double f = 1.0 + a.s * a.U * chi;
        for (int ii = threadIdx.x; ii < N; ii += blockDim.x) {
            const size_t ci = (size_t)q + (size_t)a.nq * (ii + (size_t)N * w);
            a.gam[ci] = cdiv(B[ii * ld + N], cscale(a.chi0[ci], f));
        }
        __syncthreads();
    }
}

__global__ void k_compact_flags(const int32_t* flags, int n, int32_t* list, int32_t* count) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        if (flags[e] != 0) {
            const int pos = atomicAdd(count, 1);
            list[pos] = e;
        }
    }
}
__global__ void k_count_flags(const int32_t* flags, int n, int32_t* count) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x)
        if (flags[e] != 0) atomicAdd(count, 1);
}

template <int N, int H, typename TF, int MODE>
int run_gj(ldga_ctx* ctx, const BseArgs& a0) {
    BseArgs a = a0;
    using V = typename C2<TF>::T;
    const int threads = ((N * H + 31) / 32) * 32;
    const size_t sm = (size_t)N * N * sizeof(double2) + 2 * (N + 1) * sizeof(V) + N * sizeof(double2) +
                      32 * sizeof(double) + N * sizeof(V) + 64;
    auto kern = k_bse_gj<N, H, TF, MODE>;
    LDGA_CUDA(ctx, set_smem(ctx, kern, sm));
    // q chunk: enough CTAs for several waves, but reuse Gamma(w) for many q
    int chunk = 8;
    while (chunk > 1 && (long)((a.nq + chunk - 1) / chunk) * a.nw < 8 * 148) chunk /= 2;
    a.qchunk = chunk;
    dim3 grid((a.nq + chunk - 1) / chunk, a.nw);
    StageTimer st_(ctx, LDGA_STAGE_BSE);
    kern<<<grid, threads, sm, ctx->stream>>>(a);
    LDGA_LAUNCHED(ctx, "k_bse_gj");
    return LDGA_OK;
}

template <int N, int H, int H32>
int run_mode(ldga_ctx* ctx, const BseArgs& a) {
    switch (ctx->prec) {
        case LDGA_PREC_FP64_INV: return run_gj<N, H, double, LDGA_PREC_FP64_INV>(ctx, a);
        case LDGA_PREC_FP64: return run_gj<N, H, double, LDGA_PREC_FP64>(ctx, a);
        default: return run_gj<N, H32, float, LDGA_PREC_MIXED>(ctx, a);
    }
}

}  // namespace

bool bse_has_fast_path(int nnu) {
    switch (nnu) {
        case 4: case 6: case 8: case 10: case 12: case 16: case 20: case 30: case 40: case 60: return true;
        default: return false;
    }
}

int launch_bse(ldga_ctx* ctx, int channel, int32_t* d_fail) {
    BseArgs a;
    a.nq = ctx->Nq; a.nnu = ctx->Nnu; a.nw = ctx->Nw; a.qchunk = 1;
    a.beta = ctx->mp.beta; a.U = ctx->mp.U;
    a.s = channel == LDGA_CH_D ? -1 : 1;
    a.Gamma = ctx->d_Gamma[channel];
    a.chi0 = ctx->d_chi0;
    a.chi = ctx->d_chi[channel];
    a.gam = ctx->d_gam[channel];
    a.flags = ctx->d_flags;
    const int n = ctx->Nq * ctx->Nw;
    int st = LDGA_OK;
    bool generic = false;
    switch (ctx->Nnu) {
        case 4: st = run_mode<4, 1, 1>(ctx, a); break;
        case 6: st = run_mode<6, 1, 1>(ctx, a); break;
        case 8: st = run_mode<8, 1, 1>(ctx, a); break;
        case 10: st = run_mode<10, 1, 1>(ctx, a); break;
        case 12: st = run_mode<12, 1, 1>(ctx, a); break;
        case 16: st = run_mode<16, 2, 1>(ctx, a); break;
        case 20: st = run_mode<20, 2, 1>(ctx, a); break;
        case 30: st = run_mode<30, 2, 2>(ctx, a); break;
        case 40: st = run_mode<40, 2, 2>(ctx, a); break;
        case 60: st = run_mode<60, 4, 2>(ctx, a); break;
        default: generic = true; break;
    }
    if (st != LDGA_OK) return st;
    const size_t smp = (size_t)ctx->Nnu * (ctx->Nnu + 1) * sizeof(double2) + 64 * sizeof(double) + 16;
    if (smp > 220 * 1024) return ctx_fail(ctx, LDGA_ERR_ARG, "fermionic box too large for the BSE kernels");
    LDGA_CUDA(ctx, set_smem(ctx, k_bse_lu_pivot, smp));
    if (generic) {
        StageTimer st_(ctx, LDGA_STAGE_BSE_FALLBACK);
        k_bse_lu_pivot<<<4 * 148, 256, smp, ctx->stream>>>(a, nullptr, n, nullptr);
        LDGA_LAUNCHED(ctx, "k_bse_lu_pivot");
    } else {
        // flagged matrices: compacted on the device, re-solved by a grid-stride pivoted kernel that reads
        // the count from device memory (zero work when nothing was flagged)
        LDGA_CUDA(ctx, cudaMemsetAsync(ctx->d_count, 0, sizeof(int32_t), ctx->stream));
        k_compact_flags<<<148, 256, 0, ctx->stream>>>(ctx->d_flags, n, ctx->d_list, ctx->d_count);
        LDGA_LAUNCHED(ctx, "k_compact_flags");
        StageTimer st_(ctx, LDGA_STAGE_BSE_FALLBACK);
        k_bse_lu_pivot<<<2 * 148, 256, smp, ctx->stream>>>(a, ctx->d_list, 0, ctx->d_count);
        LDGA_LAUNCHED(ctx, "k_bse_lu_pivot");
    }
    // matrices that stayed non-finite after the pivoted solve, accumulated into *d_fail
    k_count_flags<<<148, 256, 0, ctx->stream>>>(ctx->d_flags, n, d_fail);
    LDGA_LAUNCHED(ctx, "k_count_flags");
    return LDGA_OK;
}
