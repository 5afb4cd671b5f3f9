// a7: batched Bethe-Salpeter solve (calc_χγ, BSETools.jl:192-248; inv! LapackWrapper.jl:64-72).
//
// For every (q, w) the reference inverts A = Gamma_r(w) + diag(1/chi0(q, :, w)) with zgetrf+zgetri
// and only uses y = (1^T A^-1)^T, i.e. the solution of B y = 1 with B = A^T:
//     chi_r(q, w) = Re(sum_nu y_nu) / beta^2,   gamma_r(q, nu, w) = y_nu / (chi0(q,nu,w)(1 + s U chi_r)).
//
// Layout.  One CTA per (w, chunk of q); Gamma(w) is staged once in shared memory (FP64) and shared
// by MPC independent matrix groups.  A group of TR x TC threads owns one matrix [B | 1] (N rows,
// N + 1 columns) as a 2D cyclic register tile: thread (tr, tc) holds rows tr + TR*a and columns
// tc + TC*c.  The TC threads of a row group are adjacent lanes of one warp.
//
// Gauss-Jordan step k (unrolled; every register index is static):
//   1. the row group of row k writes its part of row k (columns >= k) to a double-buffered shared
//      row; the owner of the pivot also writes the pivot's reciprocal (FP32 rcp seed + two FP64
//      Newton steps: no IEEE divide on the critical path);
//   2. one named barrier over the group's threads (other groups of the CTA run on);
//   3. in every row group the lane owning column k forms the multipliers m = b_ik / b_kk of its rows
//      and shuffles them to the other lanes of the group, which update their columns > k.
// The multipliers replace the eliminated column (kept for refinement).  Work is ~N^3/2 complex
// multiply-adds: only the tile column that straddles k carries a runtime predicate.
//
// Modes:
//   LDGA_PREC_FP64_INV  in-place FP64 Gauss-Jordan inverse (N^3, the reference's formulation);
//                       y = row sums of B^-1.
//   LDGA_PREC_FP64      FP64 elimination of [B | 1].
//   LDGA_PREC_MIXED     per box size the fastest of: the q-shared preconditioned iteration
//                       (k_bse_iter: an FP32 inverse per group of 32 q, FP64 residual sweeps; at
//                       Nν = 40 both products on tensor cores: FP64 mma.sync m8n8k4 for the residual,
//                       TF32 m16n8k8 for the correction), an FP32 elimination with FP64
//                       iterative refinement (r = 1 - B y in FP64, the correction from the stored
//                       FP32 multipliers), or the FP64 elimination.
// No pivoting is done in the fast path.  Every solution is verified by its FP64 backward error
// |1 - B y|_inf / (|B|_inf |y|_inf + 1); a matrix above 1e-12 (1e-14 for the preconditioned
// iteration), or with a non-finite y, is flagged
// and re-solved by a partial-pivoting FP64 LU kernel, which is also the path for box sizes that
// have no tiled instantiation.
#include <cmath>
#include <map>
#include <mutex>

#include "ldga_internal.cuh"
#include "ns_inverse.cuh"

#ifndef LDGA_LU_LOOKAHEAD
#define LDGA_LU_LOOKAHEAD true
#endif

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
// 1/z = conj(z)/|z|^2, 1/|z|^2 from an FP32 rcp seed refined by Newton steps (FP64: two steps,
// relative error ~ seed^4, below rounding).  |z|^2 outside the FP32 range gives a non-finite
// result, which the backward-error check routes to the pivoted FP64 path.
__device__ __forceinline__ double2 vinv(double2 z) {
    const double d = z.x * z.x + z.y * z.y;
    double r = (double)__frcp_rn((float)d);
    double e = fma(-d, r, 1.0);
    r = fma(r, e, r);
    e = fma(-d, r, 1.0);
    r = fma(r, e, r);
    return make_double2(z.x * r, -z.y * r);
}
__device__ __forceinline__ float2 vinv(float2 z) {
    const float d = z.x * z.x + z.y * z.y;
    const float r = __frcp_rn(d);
    return make_float2(z.x * r, -z.y * r);
}

template <typename V>
__device__ __forceinline__ V shfl_v(V v, int src) {
    V r;
    r.x = __shfl_sync(0xffffffffu, v.x, src);
    r.y = __shfl_sync(0xffffffffu, v.y, src);
    return r;
}

__device__ __forceinline__ void named_barrier(int id, int nthreads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

struct BseArgs {
    int nq, nnu, nw, qchunk;
    double beta, U;
    int s;                  // -1 for d, +1 for m
    const double2* Gamma;   // [Nnu, Nnu, Nw]
    const double2* chi0;    // [Nq, Nnu, Nw]
    double* chi;            // [Nq, Nw]
    double2* gam;           // [Nq, Nnu, Nw]
    int32_t* flags;         // [Nq, Nw]
    unsigned long long* stats = nullptr;   // [2] k_bse_iter: residual passes and warps (may be null)
    // k_bse_iter: a flagged matrix is also appended (q + Nq w) to fail_list at atomicAdd(fail_count)
    int32_t* fail_list = nullptr;
    int32_t* fail_count = nullptr;
    int max_sweeps = 40;    // k_bse_iter: residual sweeps before a q is flagged
    // k_bse_iter<..., ADJ = true>: right-hand sides [Nq, NL, Nw] instead of ones; the conjugate of the
    // solution goes to gam (which may be rhs itself), chi is not written
    const double2* rhs = nullptr;
};

__device__ __forceinline__ double2 dmk(double r, double i) { return make_double2(r, i); }

// Group-wide reduction of NV values (op 1: max, 0: sum) over the group's G threads, fixed order.
// red: per-group shared scratch [NV * (G/32)].  Result in every thread of the group.
template <int NV, int G>
__device__ __forceinline__ void group_reduce(double (&v)[NV], const int (&op)[NV], double* red, int bar_id,
                                             int t) {
    constexpr int NWG = G / 32;
    const int wg = t >> 5, l = t & 31;
#pragma unroll
    for (int j = 0; j < NV; ++j)
        for (int o = 16; o > 0; o >>= 1) {
            const double x = __shfl_down_sync(0xffffffffu, v[j], o);
            v[j] = op[j] ? fmax(v[j], x) : v[j] + x;
        }
    named_barrier(bar_id, G);   // previous readers of red are done
    if (l == 0) {
#pragma unroll
        for (int j = 0; j < NV; ++j) red[j * NWG + wg] = v[j];
    }
    named_barrier(bar_id, G);
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        double r = 0.0;
        for (int i = 0; i < NWG; ++i) r = op[j] ? fmax(r, red[j * NWG + i]) : r + red[j * NWG + i];
        v[j] = r;
    }
}

template <int N, int TR, int TC>
struct Tile {
    static constexpr int RT = (N + TR - 1) / TR;          // tile rows
    static constexpr int NC = N + 1;                      // columns incl. the right-hand side
    static constexpr int CT = (NC + TC - 1) / TC;         // tile columns
    static constexpr int G = TR * TC;                     // threads per matrix group
    static constexpr int RW = N + 2;                      // published row: columns, rhs, reciprocal
};

template <int N, int TR, int TC, typename V>
constexpr size_t group_smem() {
    using T = Tile<N, TR, TC>;
    // rowbuf [2][RW] V, pinv [N] V, rk [2] V, ysm [N] double2, red [8 * G/32] double
    return 2 * T::RW * sizeof(V) + N * sizeof(V) + 2 * sizeof(V) + N * sizeof(double2) +
           8 * (T::G / 32) * sizeof(double) + 16;
}

// MINB: resident CTAs per SM the register allocation must allow
template <int N, int TR, int TC, int MPC, int MINB, typename TF, int MODE>
__global__ void __launch_bounds__(TR * TC * MPC, MINB) k_bse_tile(const BseArgs a) {
    using V = typename C2<TF>::T;
    using TL = Tile<N, TR, TC>;
    static_assert(TR == TC, "the blocked elimination needs a square thread grid");
    constexpr int T = TC;
    constexpr int RT = TL::RT, CT = TL::CT, G = TL::G, RW = TL::RW;
    constexpr bool MIXED = MODE == LDGA_PREC_MIXED;
    constexpr bool INV = MODE == LDGA_PREC_FP64_INV;
    constexpr int TCN = N % TC, CN = N / TC;              // owner lane / slot of the rhs column
    extern __shared__ double2 sm[];
    double2* Gsm = sm;                                    // [N*N] Gamma(w), G[j + N*i]
    const int tid = threadIdx.x;
    const int g = tid / G, t = tid - g * G;
    const int tr = t / TC, tc = t - (t / TC) * TC;
    const int lane = tid & 31;
    const int gbase = lane - tc;                          // first lane of this row group
    const int bar = g + 1;
    char* gs = reinterpret_cast<char*>(Gsm + N * N) + g * group_smem<N, TR, TC, V>();
    V* rowbuf = reinterpret_cast<V*>(gs);                 // [2][RW]
    V* pinv = rowbuf + 2 * RW;                            // [N]
    V* rkbuf = pinv + N;                                  // [2]
    double2* ysm = reinterpret_cast<double2*>(rkbuf + 2); // [N]
    double* red = reinterpret_cast<double*>(ysm + N);     // [8 * G/32]

    const int w = blockIdx.y;
    const int q0 = blockIdx.x * a.qchunk;
    const int q1 = min(a.nq, q0 + a.qchunk);
    {
        const double2* Gw = a.Gamma + (size_t)w * N * N;
        for (int e = tid; e < N * N; e += blockDim.x) Gsm[e] = Gw[e];
    }
    __syncthreads();

    for (int q = q0 + g; q < q1; q += MPC) {
        const double2* c0p = a.chi0 + (size_t)q + (size_t)a.nq * ((size_t)N * w);
        // ---- load the tile of [B | 1], B_ij = Gamma[j, i] + delta_ij / chi0(q, i, w)
        V b[RT][CT];
#pragma unroll
        for (int ra = 0; ra < RT; ++ra) {
            const int i = tr + TR * ra;
#pragma unroll
            for (int c = 0; c < CT; ++c) {
                const int j = tc + TC * c;
                double2 v = dmk(0.0, 0.0);
                if (i < N) {
                    if (j < N) {
                        v = Gsm[i * N + j];
                        if (j == i) v = cadd(v, cinv(c0p[(size_t)a.nq * i]));
                    } else if (j == N) {
                        v = dmk(1.0, 0.0);
                    }
                }
                b[ra][c] = vmk<V>(v.x, v.y);
            }
        }

        // ---- elimination.  Step k = ktc + T kc: row k is tile row kc of row group ktc and column k is
        // tile column kc of lane ktc, so kc is a compile-time index (unrolled blocks) while ktc runs
        // as an ordinary loop -- static register indices with a small code footprint.
#pragma unroll
        for (int kc = 0; kc < (N + T - 1) / T; ++kc) {
            const int kend = (N - T * kc) < T ? (N - T * kc) : T;
#pragma unroll 1
            for (int ktc = 0; ktc < kend; ++ktc) {
                const int k = ktc + T * kc;
                V* rb = rowbuf + (k & 1) * RW;
                if (tr == ktc) {
#pragma unroll
                    for (int c = 0; c < CT; ++c) {
                        const int j = tc + T * c;
                        if ((INV || c >= kc) && j <= N) rb[j] = b[kc][c];
                    }
                    if (tc == ktc) {
                        const V iv = vinv(b[kc][kc]);
                        rb[N + 1] = iv;
                        pinv[k] = iv;
                    }
                }
                named_barrier(bar, G);
                const V inv = rb[N + 1];
                if (INV) {
                    // in-place Gauss-Jordan inverse on the N x N part: row k scaled by 1/p (b_kk -> 1/p);
                    // other rows b_ij -= b_ik row_k[j] / p, b_ik -> -b_ik / p
                    V u[CT];
#pragma unroll
                    for (int c = 0; c < CT; ++c) {
                        const int j = tc + T * c;
                        u[c] = (j == k) ? inv : (j < N ? vmul<V>(rb[j], inv) : vmk<V>(0.0, 0.0));
                    }
#pragma unroll
                    for (int ra = 0; ra < RT; ++ra) {
                        V f = tc == ktc ? b[ra][kc] : vmk<V>(0.0, 0.0);
                        f = shfl_v<V>(f, gbase + ktc);
                        if (ra == kc && tr == ktc) {
#pragma unroll
                            for (int c = 0; c < CT; ++c) b[ra][c] = u[c];
                        } else {
                            if (tc == ktc) b[ra][kc] = vmk<V>(0.0, 0.0);
#pragma unroll
                            for (int c = 0; c < CT; ++c) vfnms<V>(b[ra][c], f, u[c]);
                        }
                    }
                } else {
                    V u[CT];
#pragma unroll
                    for (int c = 0; c < CT; ++c) {
                        const int j = tc + T * c;
                        if (c >= kc) u[c] = (j > k && j <= N) ? rb[j] : vmk<V>(0.0, 0.0);
                    }
#pragma unroll
                    for (int ra = 0; ra < RT; ++ra) {
                        const bool rowk = (ra == kc) && (tr == ktc);
                        V m = vmk<V>(0.0, 0.0);
                        if (tc == ktc && !rowk) {
                            m = vmul<V>(b[ra][kc], inv);
                            b[ra][kc] = m;                     // the multiplier replaces column k
                        }
                        m = shfl_v<V>(m, gbase + ktc);
                        if (!rowk) {
#pragma unroll
                            for (int c = 0; c < CT; ++c) {
                                if (c > kc || (c == kc && tc > ktc)) vfnms<V>(b[ra][c], m, u[c]);
                            }
                        }
                    }
                }
            }
        }

        // ---- solution y (FP64), shared through ysm
        double2 y[RT];
#pragma unroll
        for (int ra = 0; ra < RT; ++ra) {
            const int i = tr + TR * ra;
            if (INV) {
                double2 part = dmk(0.0, 0.0);
#pragma unroll
                for (int c = 0; c < CT; ++c) {
                    const int j = tc + TC * c;
                    if (j < N) part = cadd(part, dmk((double)b[ra][c].x, (double)b[ra][c].y));
                }
#pragma unroll
                for (int o = 1; o < TC; o <<= 1) {
                    part.x += __shfl_xor_sync(0xffffffffu, part.x, o);
                    part.y += __shfl_xor_sync(0xffffffffu, part.y, o);
                }
                y[ra] = part;
            } else {
                V z = tc == TCN ? b[ra][CN] : vmk<V>(0.0, 0.0);
                z = shfl_v<V>(z, gbase + TCN);
                const V tv = i < N ? vmul<V>(z, pinv[i]) : vmk<V>(0.0, 0.0);
                y[ra] = dmk((double)tv.x, (double)tv.y);
            }
            if (i < N && tc == 0) ysm[i] = y[ra];
        }
        named_barrier(bar, G);

        // ---- FP64 backward error (all modes) and, for MIXED, iterative refinement
        double ysum = 0.0, berr = 0.0;
        constexpr int max_ref = MIXED ? 6 : 0;
        for (int it = 0; it <= max_ref; ++it) {
            double2 r[RT];
            double st[4] = {0.0, 0.0, 0.0, 0.0};
            const int op[4] = {1, 1, 1, 0};
#pragma unroll
            for (int ra = 0; ra < RT; ++ra) {
                const int i = tr + TR * ra;
                double2 acc = dmk(0.0, 0.0);
                double rown = 0.0;
                if (i < N) {
#pragma unroll
                    for (int c = 0; c < CT; ++c) {
                        const int j = tc + TC * c;
                        if (j < N) {
                            double2 gv = Gsm[i * N + j];
                            if (j == i) gv = cadd(gv, cinv(c0p[(size_t)a.nq * i]));
                            acc = cadd(acc, cmul(gv, ysm[j]));
                            rown += fabs(gv.x) + fabs(gv.y);
                        }
                    }
                }
#pragma unroll
                for (int o = 1; o < TC; o <<= 1) {
                    acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
                    acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
                    rown += __shfl_xor_sync(0xffffffffu, rown, o);
                }
                r[ra] = i < N ? dmk(1.0 - acc.x, -acc.y) : dmk(0.0, 0.0);
                if (i < N && tc == 0) {
                    st[0] = fmax(st[0], fabs(r[ra].x) + fabs(r[ra].y));
                    st[1] = fmax(st[1], fabs(y[ra].x) + fabs(y[ra].y));
                    st[2] = fmax(st[2], rown);
                    st[3] += y[ra].x;
                }
            }
            group_reduce<4, G>(st, op, red, bar, t);
            berr = st[0] / (st[2] * st[1] + 1.0);
            ysum = st[3];
            // refinement stops once the FP64 backward error is below 1e-14 (the verification bar is 1e-12)
            if (!MIXED || it == max_ref || !isfinite(berr) || berr <= 1e-14) break;
            // correction: replay the stored FP32 elimination on r (r replicated across each row group)
            V rv[RT];
#pragma unroll
            for (int ra = 0; ra < RT; ++ra) rv[ra] = vmk<V>(r[ra].x, r[ra].y);
#pragma unroll
            for (int kc = 0; kc < (N + T - 1) / T; ++kc) {
                const int kend = (N - T * kc) < T ? (N - T * kc) : T;
#pragma unroll 1
                for (int ktc = 0; ktc < kend; ++ktc) {
                    const int k = ktc + T * kc;
                    if (tr == ktc && tc == 0) rkbuf[k & 1] = rv[kc];
                    named_barrier(bar, G);
                    const V rk = rkbuf[k & 1];
#pragma unroll
                    for (int ra = 0; ra < RT; ++ra) {
                        const bool rowk = (ra == kc) && (tr == ktc);
                        V tv = (tc == ktc && !rowk) ? vmul<V>(b[ra][kc], rk) : vmk<V>(0.0, 0.0);
                        tv = shfl_v<V>(tv, gbase + ktc);
                        if (!rowk) { rv[ra].x -= tv.x; rv[ra].y -= tv.y; }
                    }
                }
            }
#pragma unroll
            for (int ra = 0; ra < RT; ++ra) {
                const int i = tr + TR * ra;
                if (i < N) {
                    const V d = vmul<V>(rv[ra], pinv[i]);
                    y[ra] = cadd(y[ra], dmk((double)d.x, (double)d.y));
                }
            }
            named_barrier(bar, G);
#pragma unroll
            for (int ra = 0; ra < RT; ++ra) {
                const int i = tr + TR * ra;
                if (i < N && tc == 0) ysm[i] = y[ra];
            }
            named_barrier(bar, G);
        }

        // ---- chi and gamma
        const double chi = ysum / (a.beta * a.beta);
        const bool ok = isfinite(berr) && berr <= 1e-12;
        if (t == 0) {
            a.chi[(size_t)q + (size_t)a.nq * w] = chi;
            a.flags[(size_t)q + (size_t)a.nq * w] = ok ? 0 : 1;
        }
        const double f = 1.0 + a.s * a.U * chi;
#pragma unroll
        for (int ra = 0; ra < RT; ++ra) {
            const int i = tr + TR * ra;
            if (i < N && tc == 0) {
                const size_t ci = (size_t)q + (size_t)a.nq * (i + (size_t)N * w);
                a.gam[ci] = cdiv(y[ra], cscale(a.chi0[ci], f));
            }
        }
        named_barrier(bar, G);   // ysm / pinv of this matrix are read before the next one writes
    }
}

// ------------------------------------------------------------------------------------------------
// FP64 single right-hand side by LU with Gauss-Jordan inside the diagonal blocks: forward elimination
// of the rows below the pivot plus the rows above it in the same T-row block (~N^3/3 + N^2 T/2 complex
// multiply-adds instead of full Gauss-Jordan's N^3/2), then a block back substitution without any
// sequential triangular solve.
//
// Same 2-D cyclic register tile as k_bse_tile (thread (tr, tc) of a T x T group holds rows tr + T a,
// columns tc + T c of [B | 1]).  Step k = ktc + T kc:
//   1. the row group of row k shuffles the pivot b_kk from lane ktc, forms 1/b_kk (FP32 rcp seed +
//      two FP64 Newton steps) and writes row k scaled by it (columns >= T kc) to a double-buffered
//      shared row; the lanes owning column k write column k (rows >= T kc) to a double-buffered
//      shared column;
//   2. one named barrier per matrix group;
//   3. every thread updates its tile rows >= kc except row k (so the rows of tile row kc above the
//      pivot are eliminated too: the block becomes diagonal) times its tile columns > k.  The rows
//      above the pivot in tile row kc cost no extra issue slots: that tile row is issued anyway,
//      under a runtime predicate.
// Padding rows (i >= N) and columns (j > N) hold zeros and stay zero, so no step needs a bounds
// predicate.  Both broadcasts are shared-memory reads (one 16-byte load per value).
// Back substitution, tile row r from the last to the first: every row of block r only needs the
// solution of later blocks: the row group folds its lanes' partial sums (three xor shuffles), the rhs
// lane writes y_i = (z_i - sum) / b_ii, one named barrier, and every lane adds u_ij y_j of its column
// of block r into the partial sums of the rows above.
// The solution is verified by its FP64 backward error exactly like k_bse_tile (flag above 1e-12).
template <int N, int T>
struct LuSmem {
    static constexpr int RT = (N + T - 1) / T;
    static constexpr int NC = N + 1;
    static constexpr int CT = (NC + T - 1) / T;
    static constexpr int G = T * T;
    static constexpr int RW = CT * T;   // published row, padded to whole tile columns
    static constexpr int CW = RT * T;   // published column, padded to whole tile rows
    // rowbuf [2][RW], colbuf [2][CW], pinv [N], dinv [N], ysm [N] (double2), red [8 * G/32] (double)
    static constexpr size_t bytes =
        (2 * RW + 2 * CW + N + N + N) * sizeof(double2) + 8 * (G / 32) * sizeof(double) + 16;
};

template <int N, int T, int MPC, int MINB, bool GSM, bool LA>
__global__ void __launch_bounds__(T * T * MPC, MINB) k_bse_lu(const BseArgs a) {
    using LS = LuSmem<N, T>;
    constexpr int RT = LS::RT, NC = LS::NC, G = LS::G;
    constexpr int CT = (NC + T - 1) / T;
    constexpr int TCN = N % T, CN = N / T;                // owner lane / tile column of the rhs
    static_assert(T <= 32 && 32 % T == 0, "a row group must sit inside one warp");
    extern __shared__ double2 sm[];
    // Gamma(w): staged in shared memory (GSM), or read through L1/L2 when N x N does not fit
    const double2* Gsm = GSM ? sm : a.Gamma + (size_t)blockIdx.y * N * N;   // Gamma[j + N*i] at i*N + j
    const int tid = threadIdx.x;
    const int g = tid / G, t = tid - g * G;
    const int tr = t / T, tc = t - (t / T) * T;
    const int lane = tid & 31;
        const int bar = g + 1;
    char* gs = reinterpret_cast<char*>(sm + (GSM ? N * N : 0)) + g * LS::bytes;
    double2* rowbuf = reinterpret_cast<double2*>(gs);     // [2][RW]
    double2* colbuf = rowbuf + 2 * LS::RW;                // [2][CW]
    double2* pinv = colbuf + 2 * LS::CW;                  // [N] 1/b_kk
    double2* dinv = pinv + N;                             // [N] 1/chi0(q, i, w)
    double2* ysm = dinv + N;                              // [N]
    double* red = reinterpret_cast<double*>(ysm + N);     // [8 * G/32]

    const int w = blockIdx.y;
    const int q0 = blockIdx.x * a.qchunk;
    const int q1 = min(a.nq, q0 + a.qchunk);
    if (GSM) {
        const double2* Gw = a.Gamma + (size_t)w * N * N;
        for (int e = tid; e < N * N; e += blockDim.x) sm[e] = Gw[e];
    }
    __syncthreads();

    for (int q = q0 + g; q < q1; q += MPC) {
        const double2* c0p = a.chi0 + (size_t)q + (size_t)a.nq * ((size_t)N * w);
        for (int i = t; i < N; i += G) dinv[i] = cinv(c0p[(size_t)a.nq * i]);
        named_barrier(bar, G);
        // ---- load the tile of [B | 1], B_ij = Gamma[j, i] + delta_ij / chi0(q, i, w); the diagonal
        // i == j can only fall into tile (ra, ra) of the threads with tr == tc
        double2 b[RT][CT];
#pragma unroll
        for (int ra = 0; ra < RT; ++ra) {
            const int i = tr + T * ra;
#pragma unroll
            for (int c = 0; c < CT; ++c) {
                const int j = tc + T * c;
                double2 v = dmk(0.0, 0.0);
                if (i < N) {
                    if (j < N) {
                        v = Gsm[i * N + j];
                        if (c == ra && tr == tc) v = cadd(v, dinv[i]);
                    } else if (j == N) {
                        v = dmk(1.0, 0.0);
                    }
                }
                b[ra][c] = v;
            }
        }

        // ---- forward elimination (rows below the pivot).  Padding rows (i >= N) and columns (j > N)
        // of the tile hold zeros and stay zero (their published values are zero), so no step needs
        // a bounds predicate; entries at or left of the pivot are published but never read.
        const unsigned gmask = (T == 32 ? 0xffffffffu : ((1u << T) - 1u)) << (lane & ~(T - 1));
        if constexpr (LA) {
            // Lookahead: in step k every thread first updates its part of the tile row and tile
            // column that hold row k+1 and column k+1, the owners then publish step k+1 into the other
            // buffer pair, and only then is the rest of the tile updated, so the pivot shuffle, the
            // reciprocal and the stores of step k+1 overlap the bulk of step k.  Writing buffer
            // (k+1)&1 after barrier k is safe: its last readers (step k-1) finished before barrier k.
            // publish(kp, ktp): step kp = ktp + T kp (kp a compile-time tile index)
#define LDGA_LU_PUBLISH(KP, KTP)                                                                  \
            {                                                                                   \
                const int kk_ = (KTP) + T * (KP);                                                \
                double2* rb_ = rowbuf + (kk_ & 1) * LS::RW;                                      \
                double2* cb_ = colbuf + (kk_ & 1) * LS::CW;                                      \
                if (tr == (KTP)) {                                                               \
                    double2 p_;                                                                  \
                    p_.x = __shfl_sync(gmask, b[KP][KP].x, (KTP), T);                            \
                    p_.y = __shfl_sync(gmask, b[KP][KP].y, (KTP), T);                            \
                    const double2 inv_ = vinv(p_);                                               \
                    if (tc == (KTP)) pinv[kk_] = inv_;                                           \
                    _Pragma("unroll") for (int c_ = (KP); c_ < CT; ++c_)                         \
                        rb_[tc + T * c_] = vmul<double2>(b[KP][c_], inv_);                       \
                }                                                                                \
                if (tc == (KTP)) {                                                               \
                    _Pragma("unroll") for (int r_ = (KP); r_ < RT; ++r_) cb_[tr + T * r_] = b[r_][KP]; \
                }                                                                                \
            }
            // update of step k (tile index KC, lane ktc) restricted to the elements with COND(ra, c)
#define LDGA_LU_UPDATE(KC, COND)                                                                  \
            _Pragma("unroll") for (int ra = (KC); ra < RT; ++ra) {                               \
                if (ra > (KC) || tr != ktc) {                                                    \
                    const double2 m = cb[tr + T * ra];                                           \
                    _Pragma("unroll") for (int c = (KC); c < CT; ++c) {                          \
                        if ((COND) && (c > (KC) || tc > ktc)) vfnms<double2>(b[ra][c], m, u[c]); \
                    }                                                                            \
                }                                                                                \
            }
            LDGA_LU_PUBLISH(0, 0)
            named_barrier(bar, G);
#pragma unroll
            for (int kc = 0; kc < RT; ++kc) {
                const int kend = (N - T * kc) < T ? (N - T * kc) : T;
                // steps whose successor lies in the same diagonal block (cross = tile row/column kc)
#pragma unroll 1
                for (int ktc = 0; ktc < kend - 1; ++ktc) {
                    const int k = ktc + T * kc;
                    const double2* rb = rowbuf + (k & 1) * LS::RW;
                    const double2* cb = colbuf + (k & 1) * LS::CW;
                    double2 u[CT];
#pragma unroll
                    for (int c = kc; c < CT; ++c) u[c] = rb[tc + T * c];
                    LDGA_LU_UPDATE(kc, (ra == kc || c == kc))
                    LDGA_LU_PUBLISH(kc, ktc + 1)
                    LDGA_LU_UPDATE(kc, (ra != kc && c != kc))
                    named_barrier(bar, G);
                }
                // the last step of the block: the next pivot opens block kc + 1
                {
                    const int ktc = kend - 1;
                    const int k = ktc + T * kc;
                    const double2* rb = rowbuf + (k & 1) * LS::RW;
                    const double2* cb = colbuf + (k & 1) * LS::CW;
                    double2 u[CT];
#pragma unroll
                    for (int c = kc; c < CT; ++c) u[c] = rb[tc + T * c];
                    if (kc + 1 < RT) {
                        LDGA_LU_UPDATE(kc, (ra == kc + 1 || c == kc + 1))
                        LDGA_LU_PUBLISH(kc + 1, 0)
                        LDGA_LU_UPDATE(kc, (ra != kc + 1 && c != kc + 1))
                        named_barrier(bar, G);
                    } else {
                        LDGA_LU_UPDATE(kc, true)
                    }
                }
            }
#undef LDGA_LU_PUBLISH
#undef LDGA_LU_UPDATE
        } else {
    #pragma unroll
            for (int kc = 0; kc < RT; ++kc) {
                const int kend = (N - T * kc) < T ? (N - T * kc) : T;
    #pragma unroll 1
                for (int ktc = 0; ktc < kend; ++ktc) {
                    const int k = ktc + T * kc;
                    double2* rb = rowbuf + (k & 1) * LS::RW;
                    double2* cb = colbuf + (k & 1) * LS::CW;
                    if (tr == ktc) {
                        // the row group of row k scales its row by 1/b_kk (pivot shuffled from lane ktc)
                        double2 p;
                        p.x = __shfl_sync(gmask, b[kc][kc].x, ktc, T);
                        p.y = __shfl_sync(gmask, b[kc][kc].y, ktc, T);
                        const double2 inv = vinv(p);
                        if (tc == ktc) pinv[k] = inv;
    #pragma unroll
                        for (int c = kc; c < CT; ++c) rb[tc + T * c] = vmul<double2>(b[kc][c], inv);
                    }
                    if (tc == ktc) {
    #pragma unroll
                        for (int ra = kc; ra < RT; ++ra) cb[tr + T * ra] = b[ra][kc];
                    }
                    named_barrier(bar, G);
                    double2 u[CT];
    #pragma unroll
                    for (int c = kc; c < CT; ++c) u[c] = rb[tc + T * c];
    #pragma unroll
                    for (int ra = kc; ra < RT; ++ra) {
                        if (ra > kc || tr != ktc) {
                            const double2 m = cb[tr + T * ra];
    #pragma unroll
                            for (int c = kc; c < CT; ++c) {
                                if (c > kc || tc > ktc) vfnms<double2>(b[ra][c], m, u[c]);
                            }
                        }
                    }
                }
            }
        }

        // ---- back substitution, one diagonal block (tile row) at a time from the bottom
        double2 acc[RT];
#pragma unroll
        for (int ra = 0; ra < RT; ++ra) acc[ra] = dmk(0.0, 0.0);
#pragma unroll
        for (int r = RT - 1; r >= 0; --r) {
            const int nb = (N - T * r) < T ? (N - T * r) : T;
            double2 s = acc[r];
#pragma unroll
            for (int o = 1; o < T; o <<= 1) {
                s.x += __shfl_xor_sync(0xffffffffu, s.x, o);
                s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
            }
            if (tc == TCN && tr < nb) ysm[T * r + tr] = cmul(csub(b[r][CN], s), pinv[T * r + tr]);
            named_barrier(bar, G);
            if (r > 0 && T * r + tc < N) {
                const double2 yj = ysm[T * r + tc];
#pragma unroll
                for (int ra = 0; ra < r; ++ra) acc[ra] = cadd(acc[ra], cmul(b[ra][r], yj));
            }
        }

        // ---- FP64 backward error |1 - B y| / (|B| |y| + 1)
        double2 y[RT];
#pragma unroll
        for (int ra = 0; ra < RT; ++ra) {
            const int i = tr + T * ra;
            y[ra] = i < N ? ysm[i] : dmk(0.0, 0.0);
        }
        double st[4] = {0.0, 0.0, 0.0, 0.0};
        const int op[4] = {1, 1, 1, 0};
#pragma unroll
        for (int ra = 0; ra < RT; ++ra) {
            const int i = tr + T * ra;
            double2 accr = dmk(0.0, 0.0);
            double rown = 0.0;
            if (i < N) {
#pragma unroll
                for (int c = 0; c < CT; ++c) {
                    const int j = tc + T * c;
                    if (j < N) {
                        double2 gv = Gsm[i * N + j];
                        if (c == ra && tr == tc) gv = cadd(gv, dinv[i]);
                        accr = cadd(accr, cmul(gv, ysm[j]));
                        rown += fabs(gv.x) + fabs(gv.y);
                    }
                }
            }
#pragma unroll
            for (int o = 1; o < T; o <<= 1) {
                accr.x += __shfl_xor_sync(0xffffffffu, accr.x, o);
                accr.y += __shfl_xor_sync(0xffffffffu, accr.y, o);
                rown += __shfl_xor_sync(0xffffffffu, rown, o);
            }
            if (i < N && tc == 0) {
                st[0] = fmax(st[0], fabs(1.0 - accr.x) + fabs(accr.y));
                st[1] = fmax(st[1], fabs(y[ra].x) + fabs(y[ra].y));
                st[2] = fmax(st[2], rown);
                st[3] += y[ra].x;
            }
        }
        group_reduce<4, G>(st, op, red, bar, t);
        const double berr = st[0] / (st[2] * st[1] + 1.0);

        // ---- chi and gamma = y / (chi0 (1 + s U chi))
        const double chi = st[3] / (a.beta * a.beta);
        const bool ok = isfinite(berr) && berr <= 1e-12;
        if (t == 0) {
            a.chi[(size_t)q + (size_t)a.nq * w] = chi;
            a.flags[(size_t)q + (size_t)a.nq * w] = ok ? 0 : 1;
        }
        const double rf = 1.0 / (1.0 + a.s * a.U * chi);
#pragma unroll
        for (int ra = 0; ra < RT; ++ra) {
            const int i = tr + T * ra;
            if (i < N && tc == 0) {
                const size_t ci = (size_t)q + (size_t)a.nq * (i + (size_t)N * w);
                a.gam[ci] = cscale(cmul(y[ra], dinv[i]), rf);
            }
        }
        named_barrier(bar, G);   // shared buffers of this matrix are read before the next one writes
    }
}

// ------------------------------------------------------------------------------------------------
// MIXED: the k_bse_lu elimination in FP32 on packed f32x2 FMAs, then FP64 iterative refinement.
//
// A complex value of the tile is one 64-bit register pair (re, im).  b -= m u costs two f32x2 FMAs:
//     b = fma2((m.x, m.x), (-u.x, -u.y), b);   b = fma2((m.y, m.y), (u.y, -u.x), b)
// The publishing threads store both operands pre-arranged, so every broadcast is one 16-byte
// shared-memory load: the pivot row as (-u.x, -u.y, u.y, -u.x) per column, the pivot column as
// (m.x, m.x, m.y, m.y) per row.
//
// Refinement (all modes verify with the same FP64 backward error):
//   r = 1 - B y in FP64 (Gamma from shared memory, 1/chi0 in FP64);
//   forward replay of the stored FP32 elimination on r: z_i -= b_ik z_k / b_kk for the same rows
//   as step k (the elimination leaves column k of every row it touched holding b_ik), one named
//   barrier per step, z in shared memory;
//   block back substitution with the stored U exactly like the first solve;  y += delta (FP64).
// It stops once the backward error is below 1e-14; the flag threshold is 1e-12 as everywhere.
typedef unsigned long long f2p;
__device__ __forceinline__ f2p p2(float x, float y) {
    f2p r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(x), "f"(y));
    return r;
}
__device__ __forceinline__ float2 u2(f2p v) {
    float2 r;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(v));
    return r;
}
__device__ __forceinline__ f2p fma2(f2p a, f2p b, f2p c) {
    f2p d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ float2 finv(float2 z) {
    const float r = __frcp_rn(z.x * z.x + z.y * z.y);
    return make_float2(z.x * r, -z.y * r);
}

template <int N, int T>
struct Lu32Smem {
    static constexpr int RT = (N + T - 1) / T;
    static constexpr int CT = (N + 1 + T - 1) / T;
    static constexpr int G = T * T;
    static constexpr int RW = CT * T;
    static constexpr int CW = RT * T;
    // rowbuf [2][RW] float4, colbuf [2][CW] float4, pinv [N] float2, zsm [RT*T] float2,
    // dinv [N] double2, ysm [N] double2, red [8 * G/32] double
    static constexpr size_t bytes = (2 * RW + 2 * CW) * sizeof(float4) + (N + RT * T) * sizeof(float2) +
                                    2 * N * sizeof(double2) + 8 * (G / 32) * sizeof(double) + 16;
};

template <int N, int T, int MPC, int MINB, bool GSM>
__global__ void __launch_bounds__(T * T * MPC, MINB) k_bse_lu32(const BseArgs a) {
    using LS = Lu32Smem<N, T>;
    constexpr int RT = LS::RT, CT = LS::CT, G = LS::G;
    constexpr int TCN = N % T, CN = N / T;                // owner lane / tile column of the rhs
    constexpr int MAX_REF = 6;
    static_assert(T <= 32 && 32 % T == 0, "a row group must sit inside one warp");
    static_assert((N * N * sizeof(double2)) % 16 == 0, "16-byte alignment of the group buffers");
    extern __shared__ double2 sm[];
    // Gamma(w): staged in shared memory (GSM), or read through L1/L2 when N x N does not fit
    const double2* Gsm = GSM ? sm : a.Gamma + (size_t)blockIdx.y * N * N;   // Gamma[j + N*i] at i*N + j
    const int tid = threadIdx.x;
    const int g = tid / G, t = tid - g * G;
    const int tr = t / T, tc = t - (t / T) * T;
    const int lane = tid & 31;
    const int bar = g + 1;
    char* gs = reinterpret_cast<char*>(sm + (GSM ? N * N : 0)) + g * LS::bytes;
    float4* rowbuf = reinterpret_cast<float4*>(gs);       // [2][RW]
    float4* colbuf = rowbuf + 2 * LS::RW;                 // [2][CW]
    float2* pinv = reinterpret_cast<float2*>(colbuf + 2 * LS::CW);   // [N] 1/b_kk (FP32)
    float2* zsm = pinv + N;                               // [RT*T] refinement right-hand side
    double2* dinv = reinterpret_cast<double2*>(zsm + RT * T);        // [N] 1/chi0(q, i, w)
    double2* ysm = dinv + N;                              // [N] solution (FP64)
    double* red = reinterpret_cast<double*>(ysm + N);     // [8 * G/32]

    const int w = blockIdx.y;
    const int q0 = blockIdx.x * a.qchunk;
    const int q1 = min(a.nq, q0 + a.qchunk);
    if (GSM) {
        const double2* Gw = a.Gamma + (size_t)w * N * N;
        for (int e = tid; e < N * N; e += blockDim.x) sm[e] = Gw[e];
    }
    __syncthreads();
    const unsigned gmask = (T == 32 ? 0xffffffffu : ((1u << T) - 1u)) << (lane & ~(T - 1));

    for (int q = q0 + g; q < q1; q += MPC) {
        const double2* c0p = a.chi0 + (size_t)q + (size_t)a.nq * ((size_t)N * w);
        for (int i = t; i < N; i += G) dinv[i] = cinv(c0p[(size_t)a.nq * i]);
        named_barrier(bar, G);
        // ---- FP32 tile of [B | 1]; padding rows / columns are zero and stay zero
        f2p b[RT][CT];
#pragma unroll
        for (int ra = 0; ra < RT; ++ra) {
            const int i = tr + T * ra;
#pragma unroll
            for (int c = 0; c < CT; ++c) {
                const int j = tc + T * c;
                double2 v = dmk(0.0, 0.0);
                if (i < N) {
                    if (j < N) {
                        v = Gsm[i * N + j];
                        if (c == ra && tr == tc) v = cadd(v, dinv[i]);
                    } else if (j == N) {
                        v = dmk(1.0, 0.0);
                    }
                }
                b[ra][c] = p2((float)v.x, (float)v.y);
            }
        }

        // ---- forward elimination (LU with Gauss-Jordan inside the diagonal blocks), FP32
#pragma unroll
        for (int kc = 0; kc < RT; ++kc) {
            const int kend = (N - T * kc) < T ? (N - T * kc) : T;
#pragma unroll 1
            for (int ktc = 0; ktc < kend; ++ktc) {
                const int k = ktc + T * kc;
                float4* rb = rowbuf + (k & 1) * LS::RW;
                float4* cb = colbuf + (k & 1) * LS::CW;
                if (tr == ktc) {
                    const float2 pv = u2(b[kc][kc]);
                    float2 p;
                    p.x = __shfl_sync(gmask, pv.x, ktc, T);
                    p.y = __shfl_sync(gmask, pv.y, ktc, T);
                    const float2 inv = finv(p);
                    if (tc == ktc) pinv[k] = inv;
#pragma unroll
                    for (int c = kc; c < CT; ++c) {
                        const float2 u = fmul(u2(b[kc][c]), inv);
                        rb[tc + T * c] = make_float4(-u.x, -u.y, u.y, -u.x);
                    }
                }
                if (tc == ktc) {
#pragma unroll
                    for (int ra = kc; ra < RT; ++ra) {
                        const float2 m = u2(b[ra][kc]);
                        cb[tr + T * ra] = make_float4(m.x, m.x, m.y, m.y);
                    }
                }
                named_barrier(bar, G);
                f2p un[CT], us[CT];
#pragma unroll
                for (int c = kc; c < CT; ++c) {
                    const float4 v = rb[tc + T * c];
                    un[c] = p2(v.x, v.y);
                    us[c] = p2(v.z, v.w);
                }
#pragma unroll
                for (int ra = kc; ra < RT; ++ra) {
                    if (ra > kc || tr != ktc) {
                        const float4 mv = cb[tr + T * ra];
                        const f2p mx = p2(mv.x, mv.y), my = p2(mv.z, mv.w);
#pragma unroll
                        for (int c = kc; c < CT; ++c) {
                            if (c > kc || tc > ktc) b[ra][c] = fma2(my, us[c], fma2(mx, un[c], b[ra][c]));
                        }
                    }
                }
            }
        }

        // ---- block back substitution: z in the rhs column (lane TCN, tile column CN) -> ysm.
        // sol: FP32 solution of the current block, written to dst (FP64 y, or the correction in zsm)
        auto back_substitute = [&](bool first) {
            f2p acc[RT];
#pragma unroll
            for (int ra = 0; ra < RT; ++ra) acc[ra] = p2(0.f, 0.f);
#pragma unroll
            for (int r = RT - 1; r >= 0; --r) {
                const int nb = (N - T * r) < T ? (N - T * r) : T;
                float2 s = u2(acc[r]);
#pragma unroll
                for (int o = 1; o < T; o <<= 1) {
                    s.x += __shfl_xor_sync(0xffffffffu, s.x, o);
                    s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
                }
                if (tc == TCN && tr < nb) {
                    const int i = T * r + tr;
                    const float2 z = first ? u2(b[r][CN]) : zsm[i];
                    const float2 yi = fmul(make_float2(z.x - s.x, z.y - s.y), pinv[i]);
                    zsm[i] = yi;
                }
                named_barrier(bar, G);
                if (r > 0 && T * r + tc < N) {
                    const float2 yj = zsm[T * r + tc];
                    const f2p yx = p2(yj.x, yj.x), yy = p2(yj.y, yj.y);
#pragma unroll
                    for (int ra = 0; ra < r; ++ra) {
                        // acc += b * yj:  (b.x yj.x - b.y yj.y, b.y yj.x + b.x yj.y)
                        const float2 bv = u2(b[ra][r]);
                        acc[ra] = fma2(yy, p2(-bv.y, bv.x), fma2(yx, b[ra][r], acc[ra]));
                    }
                }
            }
        };
        back_substitute(true);
        for (int i = t; i < N; i += G) {
            const float2 v = zsm[i];
            ysm[i] = dmk((double)v.x, (double)v.y);
        }
        named_barrier(bar, G);

        // ---- FP64 backward error and refinement
        double berr = 0.0, ysum = 0.0;
        for (int it = 0; it <= MAX_REF; ++it) {
            double st[4] = {0.0, 0.0, 0.0, 0.0};
            const int op[4] = {1, 1, 1, 0};
#pragma unroll
            for (int ra = 0; ra < RT; ++ra) {
                const int i = tr + T * ra;
                double2 accr = dmk(0.0, 0.0);
                double rown = 0.0;
                if (i < N) {
#pragma unroll
                    for (int c = 0; c < CT; ++c) {
                        const int j = tc + T * c;
                        if (j < N) {
                            double2 gv = Gsm[i * N + j];
                            if (c == ra && tr == tc) gv = cadd(gv, dinv[i]);
                            accr = cadd(accr, cmul(gv, ysm[j]));
                            rown += fabs(gv.x) + fabs(gv.y);
                        }
                    }
                }
#pragma unroll
                for (int o = 1; o < T; o <<= 1) {
                    accr.x += __shfl_xor_sync(0xffffffffu, accr.x, o);
                    accr.y += __shfl_xor_sync(0xffffffffu, accr.y, o);
                    rown += __shfl_xor_sync(0xffffffffu, rown, o);
                }
                if (i < N && tc == 0) {
                    const double2 yi = ysm[i];
                    const double2 ri = dmk(1.0 - accr.x, -accr.y);
                    zsm[i] = make_float2((float)ri.x, (float)ri.y);
                    st[0] = fmax(st[0], fabs(ri.x) + fabs(ri.y));
                    st[1] = fmax(st[1], fabs(yi.x) + fabs(yi.y));
                    st[2] = fmax(st[2], rown);
                    st[3] += yi.x;
                }
            }
            group_reduce<4, G>(st, op, red, bar, t);   // its barriers also publish zsm
            berr = st[0] / (st[2] * st[1] + 1.0);
            ysum = st[3];
            if (it == MAX_REF || !isfinite(berr) || berr <= 1e-14) break;
            // forward replay of the FP32 elimination on z = r
#pragma unroll
            for (int kc = 0; kc < RT; ++kc) {
                const int kend = (N - T * kc) < T ? (N - T * kc) : T;
#pragma unroll 1
                for (int ktc = 0; ktc < kend; ++ktc) {
                    const int k = ktc + T * kc;
                    if (tc == ktc) {
                        const float2 zk = fmul(zsm[k], pinv[k]);
#pragma unroll
                        for (int ra = kc; ra < RT; ++ra) {
                            const int i = tr + T * ra;
                            if (i < N && i != k) {
                                const float2 m = u2(b[ra][kc]);
                                const float2 d = fmul(m, zk);
                                float2 zi = zsm[i];
                                zi.x -= d.x; zi.y -= d.y;
                                zsm[i] = zi;
                            }
                        }
                    }
                    named_barrier(bar, G);
                }
            }
            // back substitution on the corrected rhs (reads z_i, writes delta_i into zsm)
            back_substitute(false);
            for (int i = t; i < N; i += G) {
                const float2 d = zsm[i];
                ysm[i] = cadd(ysm[i], dmk((double)d.x, (double)d.y));
            }
            named_barrier(bar, G);
        }

        // ---- chi and gamma = y / (chi0 (1 + s U chi))
        const double chi = ysum / (a.beta * a.beta);
        const bool ok = isfinite(berr) && berr <= 1e-12;
        if (t == 0) {
            a.chi[(size_t)q + (size_t)a.nq * w] = chi;
            a.flags[(size_t)q + (size_t)a.nq * w] = ok ? 0 : 1;
        }
        const double rf = 1.0 / (1.0 + a.s * a.U * chi);
        for (int i = t; i < N; i += G) {
            const size_t ci = (size_t)q + (size_t)a.nq * (i + (size_t)N * w);
            a.gam[ci] = cscale(cmul(ysm[i], dinv[i]), rf);
        }
        named_barrier(bar, G);   // shared buffers of this matrix are read before the next one writes
    }
}

// ------------------------------------------------------------------------------------------------
// MIXED, one matrix per warp: the FP32 f32x2 elimination of k_bse_lu32 and an FP64-refined solve
// without any barrier.  The warp holds [B | 1] as a TR x TC lane grid (TR * TC = 32, TR >= TC;
// lane tr * TC + tc owns rows tr + TR a and columns tc + TC c).
//
// Elimination step k (row tile k / TR and column tile k / TC are compile-time indices: the row
// tiles are unrolled, inside them the TR / TC column tiles, and only the TC steps of one column
// tile run as a loop):
//   1. the row group of row k shuffles the pivot, forms 1/b_kk and stores row k scaled by it as
//      (-u.x, -u.y, u.y, -u.x); the lanes owning column k store it as (m.x, m.x, m.y, m.y).  The
//      publishers store zeros where nothing may change (row k itself, the columns <= k of the
//      pivot's tile column), so the consumers need no predicate;
//   2. __syncwarp; every lane loads its multipliers and row values (16-byte shared loads) and
//      updates b -= m u with two f32x2 FMAs per complex element:
//          b = fma2((m.y, m.y), (u.y, -u.x), fma2((m.x, m.x), (-u.x, -u.y), b)).
// Gauss-Jordan inside the TR-row diagonal blocks (as in k_bse_lu) leaves those blocks diagonal,
// so the back substitution walks the row tiles from the bottom with one shuffle reduction each.
//
// Refinement (FP64 residual, FP32 correction from the stored factors, y += delta) until the FP64
// backward error |1 - B y|_inf / (|B|_inf |y|_inf + 1) is below 1e-14; the flag threshold for the
// pivoted FP64 fallback is 1e-12 as in every mode.  The correction's forward replay is blocked:
// per row tile, TR fully unrolled shuffle steps inside the diagonal block, then one matrix-vector
// update of all rows below (partial sums over the TC lanes of a row group, xor-shuffle reduced).
// z is replicated across the TC lanes of each row group, so no shared memory is involved.
template <int N, int TR, int TC>
struct Warp32Smem {
    static constexpr int RT = (N + TR - 1) / TR;
    static constexpr int CT = (N + 1 + TC - 1) / TC;
    // rowbuf [2][CT*TC] float4, colbuf [2][RT*TR] float4, pinv [RT*TR] float2, zsm [RT*TR] float2,
    // dinv [N] double2, ysm [N] double2
    static constexpr size_t bytes =
        (2 * CT * TC + 2 * RT * TR) * sizeof(float4) + 2 * RT * TR * sizeof(float2) + 2 * N * sizeof(double2);
};

template <int N, int TR, int TC, int WPC, int MINB>
__global__ void __launch_bounds__(32 * WPC, MINB) k_bse_warp32(const BseArgs a) {
    using WS = Warp32Smem<N, TR, TC>;
    constexpr int RT = WS::RT, CT = WS::CT;
    constexpr int NH = TR / TC;                           // tile columns per tile row
    constexpr int TCN = N % TC, CN = N / TC;              // owner lane / tile column of the rhs
    constexpr int MAX_REF = 6;
    static_assert(TR * TC == 32 && TR >= TC && TR % TC == 0, "a TR x TC lane grid filling one warp");
    extern __shared__ double2 sm[];
    double2* Gsm = sm;                                    // [N*N] Gamma(w), Gamma[j + N*i] at i*N + j
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const int tr = lane / TC, tc = lane - (lane / TC) * TC;
    char* gs = reinterpret_cast<char*>(Gsm + N * N) + wp * WS::bytes;
    float4* rowbuf = reinterpret_cast<float4*>(gs);       // [2][CT*TC]
    float4* colbuf = rowbuf + 2 * CT * TC;                // [2][RT*TR]
    float2* pinv = reinterpret_cast<float2*>(colbuf + 2 * RT * TR);  // [RT*TR] 1/b_kk (FP32)
    float2* zsm = pinv + RT * TR;                         // [RT*TR] solution of one solve
    double2* dinv = reinterpret_cast<double2*>(zsm + RT * TR);       // [N] 1/chi0(q, i, w)
    double2* ysm = dinv + N;                              // [N] solution (FP64)

    const int w = blockIdx.y;
    const int q0 = blockIdx.x * a.qchunk;
    const int q1 = min(a.nq, q0 + a.qchunk);
    {
        const double2* Gw = a.Gamma + (size_t)w * N * N;
        for (int e = threadIdx.x; e < N * N; e += blockDim.x) Gsm[e] = Gw[e];
    }
    __syncthreads();
    const unsigned rmask = (TC == 32 ? 0xffffffffu : ((1u << TC) - 1u)) << (lane & ~(TC - 1));
    const f2p zero = p2(0.f, 0.f);

    for (int q = q0 + wp; q < q1; q += WPC) {
        const double2* c0p = a.chi0 + (size_t)q + (size_t)a.nq * ((size_t)N * w);
        for (int i = lane; i < N; i += 32) dinv[i] = cinv(c0p[(size_t)a.nq * i]);
        __syncwarp();
        f2p b[RT][CT];
#pragma unroll
        for (int ra = 0; ra < RT; ++ra) {
            const int i = tr + TR * ra;
#pragma unroll
            for (int c = 0; c < CT; ++c) {
                const int j = tc + TC * c;
                double2 v = dmk(0.0, 0.0);
                if (i < N) {
                    if (j < N) {
                        v = Gsm[i * N + j];
                        if (i == j) v = cadd(v, dinv[i]);
                    } else if (j == N) {
                        v = dmk(1.0, 0.0);
                    }
                }
                b[ra][c] = p2((float)v.x, (float)v.y);
            }
        }

        // ---- forward elimination, FP32
#pragma unroll
        for (int rak = 0; rak < RT; ++rak) {
#pragma unroll
            for (int h = 0; h < NH; ++h) {
                const int k0 = TR * rak + TC * h;
                if (k0 >= N) break;
                const int ck = rak * NH + h;
                const int kend = (N - k0) < TC ? (N - k0) : TC;
#pragma unroll 1
                for (int ktc = 0; ktc < kend; ++ktc) {
                    const int k = k0 + ktc;
                    const int ktr = TC * h + ktc;
                    float4* rb = rowbuf + (k & 1) * (CT * TC);
                    float4* cb = colbuf + (k & 1) * (RT * TR);
                    // pivot to every lane; the lanes of column k scale it (RT values per lane, fewer
                    // than the CT of a row), the row group of row k stores row k unscaled
                    float2 p;
                    {
                        const float2 pv = u2(b[rak][ck]);
                        p.x = __shfl_sync(0xffffffffu, pv.x, ktr * TC + ktc);
                        p.y = __shfl_sync(0xffffffffu, pv.y, ktr * TC + ktc);
                    }
                    const float2 inv = finv(p);
                    if (tr == ktr) {
                        if (tc == ktc) pinv[k] = inv;
                        {
                            const float2 u = u2(b[rak][ck]);
                            rb[tc + TC * ck] = tc <= ktc ? make_float4(0.f, 0.f, 0.f, 0.f) : make_float4(u.x, u.y, u.y, u.x);
                        }
#pragma unroll
                        for (int c = ck + 1; c < CT; ++c) {
                            const float2 u = u2(b[rak][c]);
                            rb[tc + TC * c] = make_float4(u.x, u.y, u.y, u.x);
                        }
                    }
                    if (tc == ktc) {
                        {
                            const float2 m = fmul(u2(b[rak][ck]), inv);
                            cb[tr + TR * rak] = tr == ktr ? make_float4(0.f, 0.f, 0.f, 0.f)
                                                          : make_float4(-m.x, -m.x, m.y, -m.y);
                        }
#pragma unroll
                        for (int ra = rak + 1; ra < RT; ++ra) {
                            const float2 m = fmul(u2(b[ra][ck]), inv);
                            cb[tr + TR * ra] = make_float4(-m.x, -m.x, m.y, -m.y);
                        }
                    }
                    __syncwarp();
                    // b -= m u:  b += (-m.x, -m.x) (u.x, u.y);  b += (m.y, -m.y) (u.y, u.x)
                    f2p mx[RT], my[RT];
#pragma unroll
                    for (int ra = rak; ra < RT; ++ra) {
                        const float4 mv = cb[tr + TR * ra];
                        mx[ra] = p2(mv.x, mv.y);
                        my[ra] = p2(mv.z, mv.w);
                    }
#pragma unroll
                    for (int c = ck; c < CT; ++c) {
                        const float4 v = rb[tc + TC * c];
                        const f2p u1 = p2(v.x, v.y), u2v = p2(v.z, v.w);
#pragma unroll
                        for (int ra = rak; ra < RT; ++ra) b[ra][c] = fma2(mx[ra], u1, b[ra][c]);
#pragma unroll
                        for (int ra = rak; ra < RT; ++ra) b[ra][c] = fma2(my[ra], u2v, b[ra][c]);
                    }
                }
            }
        }

        // ---- block back substitution over the TR-row tiles: rhs z from the rhs column of the tile
        // (first solve) or from zr (replicated on the row group), FP32 solution into zsm
        float2 zr[RT];
        auto back_substitute = [&](bool first) {
            f2p acc[RT];
#pragma unroll
            for (int ra = 0; ra < RT; ++ra) acc[ra] = zero;
#pragma unroll
            for (int r = RT - 1; r >= 0; --r) {
                const int nb = (N - TR * r) < TR ? (N - TR * r) : TR;
                float2 s = u2(acc[r]);
#pragma unroll
                for (int o = 1; o < TC; o <<= 1) {
                    s.x += __shfl_xor_sync(0xffffffffu, s.x, o);
                    s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
                }
                if (tc == TCN && tr < nb) {
                    const int i = TR * r + tr;
                    const float2 z = first ? u2(b[r][CN]) : zr[r];
                    zsm[i] = fmul(make_float2(z.x - s.x, z.y - s.y), pinv[i]);
                }
                __syncwarp();
                if (r > 0) {
#pragma unroll
                    for (int c = r * NH; c < r * NH + NH; ++c) {
                        const int j = tc + TC * c;
                        if (j < TR * r + nb) {
                            const float2 yj = zsm[j];
                            const f2p yx = p2(yj.x, yj.x), yy = p2(yj.y, yj.y);
#pragma unroll
                            for (int ra = 0; ra < r; ++ra) {
                                const float2 bv = u2(b[ra][c]);
                                acc[ra] = fma2(yy, p2(-bv.y, bv.x), fma2(yx, b[ra][c], acc[ra]));
                            }
                        }
                    }
                }
            }
        };
        back_substitute(true);
        for (int i = lane; i < N; i += 32) {
            const float2 v = zsm[i];
            ysm[i] = dmk((double)v.x, (double)v.y);
        }
        __syncwarp();

        // ---- FP64 backward error and refinement
        double berr = 0.0, ysum = 0.0, bnorm = 0.0;
        for (int it = 0; it <= MAX_REF; ++it) {
            double e_r = 0.0, e_y = 0.0, sy = 0.0;
#pragma unroll
            for (int ra = 0; ra < RT; ++ra) {
                const int i = tr + TR * ra;
                double2 accr = dmk(0.0, 0.0);
                double rown = 0.0;
                if (i < N) {
#pragma unroll 1
                    for (int c = 0; c < CT; ++c) {
                        const int j = tc + TC * c;
                        if (j < N) {
                            double2 gv = Gsm[i * N + j];
                            if (i == j) gv = cadd(gv, dinv[i]);
                            const double2 yj = ysm[j];
                            accr.x = fma(gv.x, yj.x, fma(-gv.y, yj.y, accr.x));
                            accr.y = fma(gv.x, yj.y, fma(gv.y, yj.x, accr.y));
                            if (it == 0) rown += fabs(gv.x) + fabs(gv.y);
                        }
                    }
                }
#pragma unroll
                for (int o = 1; o < TC; o <<= 1) {
                    accr.x += __shfl_xor_sync(0xffffffffu, accr.x, o);
                    accr.y += __shfl_xor_sync(0xffffffffu, accr.y, o);
                    if (it == 0) rown += __shfl_xor_sync(0xffffffffu, rown, o);
                }
                const double2 ri = i < N ? dmk(1.0 - accr.x, -accr.y) : dmk(0.0, 0.0);
                zr[ra] = make_float2((float)ri.x, (float)ri.y);
                if (i < N) {
                    const double2 yi = ysm[i];
                    e_r = fmax(e_r, fabs(ri.x) + fabs(ri.y));
                    e_y = fmax(e_y, fabs(yi.x) + fabs(yi.y));
                    if (it == 0) bnorm = fmax(bnorm, rown);
                    sy += yi.x;
                }
            }
            // every lane of a row group holds its rows' values: reduce across row groups only
            // (xor over the lane bits above tc), a fixed order
#pragma unroll
            for (int o = TC; o < 32; o <<= 1) {
                e_r = fmax(e_r, __shfl_xor_sync(0xffffffffu, e_r, o));
                e_y = fmax(e_y, __shfl_xor_sync(0xffffffffu, e_y, o));
                if (it == 0) bnorm = fmax(bnorm, __shfl_xor_sync(0xffffffffu, bnorm, o));
                sy += __shfl_xor_sync(0xffffffffu, sy, o);
            }
            berr = e_r / (bnorm * e_y + 1.0);
            ysum = sy;
            if (it == MAX_REF || !isfinite(berr) || berr <= 1e-14) break;

            // forward replay of the FP32 elimination on z = r, one row tile (diagonal block) at a time
#pragma unroll
            for (int o = 0; o < RT; ++o) {
                f2p mine[NH];                     // w of the columns this lane owns in the block
#pragma unroll
                for (int h = 0; h < NH; ++h) mine[h] = zero;
#pragma unroll
                for (int s = 0; s < TR; ++s) {
                    const int k = TR * o + s;
                    if (k < N) {
                        const int h = s / TC, ktc = s % TC, ck = o * NH + h;
                        // w_k = z_k / b_kk (z_k lives on row group s)
                        float2 zk;
                        zk.x = __shfl_sync(0xffffffffu, zr[o].x, s * TC);
                        zk.y = __shfl_sync(0xffffffffu, zr[o].y, s * TC);
                        const float2 wk = fmul(zk, pinv[k]);
                        if (tc == ktc) mine[h] = p2(wk.x, wk.y);
                        // rows of the block except k: z_i -= b_ik w_k (b_ik on lane ktc of the row group)
                        float2 d = fmul(u2(b[o][ck]), wk);
                        d.x = __shfl_sync(0xffffffffu, d.x, tr * TC + ktc);
                        d.y = __shfl_sync(0xffffffffu, d.y, tr * TC + ktc);
                        if (tr != s) { zr[o].x -= d.x; zr[o].y -= d.y; }
                    }
                }
                // rows below the block: z_i -= sum_k b_ik w_k over the block's columns
#pragma unroll
                for (int ra = o + 1; ra < RT; ++ra) {
                    f2p part = zero;
#pragma unroll
                    for (int h = 0; h < NH; ++h) {
                        const float2 wv = u2(mine[h]);
                        const f2p wx = p2(wv.x, wv.x), wy = p2(wv.y, wv.y);
                        const float2 bv = u2(b[ra][o * NH + h]);
                        part = fma2(wy, p2(-bv.y, bv.x), fma2(wx, b[ra][o * NH + h], part));
                    }
                    float2 ps = u2(part);
#pragma unroll
                    for (int x = 1; x < TC; x <<= 1) {
                        ps.x += __shfl_xor_sync(0xffffffffu, ps.x, x);
                        ps.y += __shfl_xor_sync(0xffffffffu, ps.y, x);
                    }
                    zr[ra].x -= ps.x;
                    zr[ra].y -= ps.y;
                }
            }
            back_substitute(false);
            for (int i = lane; i < N; i += 32) {
                const float2 d = zsm[i];
                ysm[i] = cadd(ysm[i], dmk((double)d.x, (double)d.y));
            }
            __syncwarp();
        }

        // ---- chi and gamma = y / (chi0 (1 + s U chi))
        const double chi = ysum / (a.beta * a.beta);
        const bool ok = isfinite(berr) && berr <= 1e-12;
        if (lane == 0) {
            a.chi[(size_t)q + (size_t)a.nq * w] = chi;
            a.flags[(size_t)q + (size_t)a.nq * w] = ok ? 0 : 1;
        }
        const double rf = 1.0 / (1.0 + a.s * a.U * chi);
        for (int i = lane; i < N; i += 32) {
            const size_t ci = (size_t)q + (size_t)a.nq * (i + (size_t)N * w);
            a.gam[ci] = cscale(cmul(ysm[i], dinv[i]), rf);
        }
        __syncwarp();   // shared buffers of this matrix are read before the next one writes
    }
}

// ------------------------------------------------------------------------------------------------
// MIXED, q-shared preconditioner ("iter"; "tc": its FP32 product on tensor cores; "dm": also its
// FP64 residual product on the FP64 tensor path).  All q of one w share Gamma(w); their matrices differ only
// by the diagonal 1/chi0(q, :, w).  k_bse_qorder sorts the q of every w by
// Re 1/chi0(q, N/2 - 1, w) + Re 1/chi0(q, N/2, w), the two lowest |nu| of the box;
// a CTA of k_bse_iter takes 32 consecutive q of that order and forms, in FP32, the in-place
// Gauss-Jordan inverse C of B_bar = Gamma(w)^T + diag(mean over its q of 1/chi0).  Every q of the
// group then iterates (Richardson refinement with the approximate inverse C)
//     r = 1 - B_q x   (FP64, one N^2 product),   x += C r   (FP32 product, FP64 update)
// from x = C 1 until the FP64 backward error of x -- the measure of the LU kernels -- is at most
// 1e-14, or max_sweeps sweeps (40 unless the handle sets another); a q still above 1e-14 is flagged
// for the pivoted FP64 solve.  The
// sweep count is set by how far B_q is from B_bar (about 7 on the 3D 32^3 matrices), so the FP64
// work per matrix is ~7 N^2 instead of the elimination's N^3 / 3 plus its latency-bound steps.
// Layout: LPQ adjacent lanes per q; lane h of a q owns rows [h RPL, (h+1) RPL) of x, r and of the
// products.  x_k and r_k of the other rows come from the q's lanes by shuffles (column
// k = s RPL + j sits in lane s of the q, register j); Gamma^T and C rows are shared-memory reads
// that the LPQ distinct rows of a warp fetch in one wavefront (row stride N + 1).  Warps iterate
// independently (no CTA barrier in the loop) until all q of the warp have converged.
constexpr int kIterQ = 32;      // q per CTA: one preconditioner
constexpr int kNsMaxIts = 6;    // Newton-Schulz iterations at most (tensor-core group inverse)
constexpr float kNsTol = 1e-2f; // stop once (max row sum of |I - B_bar X|)^2 <= kNsTol
constexpr double kIterTol = 1e-14;

// TC: the FP32 product x += C r runs on tensor cores (mma.sync m16n8k8, TF32 operands, FP32
// accumulation): C is kept as the A fragments of its real and imaginary parts, MT x KT tiles of
// 16 x 8 with the rows padded to MT 16, and every warp has an exchange buffer that brings its 8 q's
// residuals into B-fragment order and the products back to the lanes that own the rows.
// DM: the FP64 residual product runs on the FP64 tensor path (mma.sync m8n8k4 .f64): Gamma^T is kept
// as the A fragments of its real and imaginary parts (N/8 x N/4 tiles of 8 x 4) instead of row-major.
// NS: the group inverse is formed by Newton-Schulz iterations on tcgen05 tensor cores
// (ns_inverse.cuh) instead of the Gauss-Jordan elimination, which stays as the fallback when the
// iteration does not converge.  Its operand buffers occupy [0, NsSmem::bytes) during the set-up,
// where the Gamma^T fragments and the C fragments / exchange buffers go afterwards, so D moves
// behind them; the mbarrier, the TMEM address and a reduction scratch follow the pivot buffers.
template <int N, bool GSM = true, bool TC = false, int NWARP = 4, bool DM = false, bool NS = false>
struct IterSmem {
    static constexpr int LD = N + 1;
    static constexpr int MT = (N + 15) / 16, KT = N / 8, XS = 2 * N + 4;   // TC tiles, exchange stride
    static constexpr int XD = N + 4;                                       // DM exchange stride (doubles)
    static constexpr size_t xw_bytes = (size_t)8 * XS * sizeof(float) > (size_t)8 * XD * sizeof(double)
                                           ? (size_t)8 * XS * sizeof(float) : (size_t)8 * XD * sizeof(double);
    static constexpr size_t c_bytes = TC ? (size_t)2 * MT * KT * 32 * 4 * sizeof(float) + (size_t)NWARP * xw_bytes
                                         : (size_t)N * LD * sizeof(float2);
    // Gt [N][LD] double2 (GSM: Gamma staged in shared memory; otherwise read through L1/L2); DM: the
    // A fragments [2][N/8][N/4][32] doubles
    static constexpr size_t g_bytes = DM ? (size_t)N * N * sizeof(double2) : GSM ? (size_t)N * LD * sizeof(double2) : 0;
    static constexpr size_t d_bytes = (size_t)kIterQ * N * sizeof(double2);      // D [32][N] double2
    static constexpr size_t ns_bytes = NS ? ns::NsSmem<(N % 8 == 0 ? N : 8)>::bytes : 0;
    static constexpr size_t c_end = g_bytes + ((c_bytes + 15) & ~size_t(15));
    static constexpr size_t off_D = NS ? (c_end > ns_bytes ? c_end : ns_bytes) : g_bytes;
    static constexpr size_t off_C = NS ? g_bytes : off_D + d_bytes;
    static constexpr size_t off_X = off_C + (TC ? (size_t)2 * MT * KT * 32 * 4 * sizeof(float) : 0);  // TC exchange
    static constexpr size_t off_rowabs = NS ? off_D + d_bytes : off_C + ((c_bytes + 15) & ~size_t(15));
    static constexpr size_t off_dbar = off_rowabs + (((size_t)N * sizeof(double) + 15) & ~size_t(15));
    // Gauss-Jordan pivot buffers [2][columns k, k+1: 2 N float2][rows k, k+1 interleaved: RW float4],
    // RW = the row width the owning threads cover (N rounded up to their segments)
    static constexpr int TPR = NWARP * 32 / N > 0 ? NWARP * 32 / N : 1;
    static constexpr int RW = (N + TPR - 1) / TPR * TPR;
    static constexpr size_t pc_half = 2 * (size_t)N * sizeof(float2) + (size_t)RW * sizeof(float4);
    static constexpr size_t off_pc = off_dbar + (size_t)N * sizeof(double2);
    // NS: mbarrier (8 bytes), TMEM address (4, padded to 8), reduction scratch [NWARP] floats
    static constexpr size_t off_bar = off_pc + 2 * pc_half, off_slot = off_bar + 8, off_red = off_bar + 16;
    static constexpr size_t bytes = NS ? off_red + ((NWARP * sizeof(float) + 15) & ~size_t(15)) : off_pc + 2 * pc_half;
    static_assert(!NS || off_bar % 8 == 0, "mbarrier alignment");
};

__device__ __forceinline__ uint32_t to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}
// d += a b, one m16n8k8 TF32 tile (a: 4 A-fragment registers, b: 2 B-fragment registers)
__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint4 a, uint32_t b0, uint32_t b1) {
    asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a.x), "r"(a.y), "r"(a.z), "r"(a.w), "r"(b0), "r"(b1));
}

// dx = C r for the warp's 8 q (lane group lane/8 holds q 2 (lane/8) + c, rows h RPL + r) on tensor
// cores.  fr / fi: A fragments of Re C / Im C, [MT][KT][32 lanes] x 4 tf32; xb: this warp's exchange
// buffer [8 q][XS] floats, (re, im) per row.  dx_re = Cr r_re - Ci r_im, dx_im = Ci r_re + Cr r_im.
template <int N, int RPL, int QPL, int LPQ>
__device__ __forceinline__ void tc_apply(const float2 (&rr)[QPL][RPL], float2 (&dx)[QPL][RPL], const uint4* fr,
                                         const uint4* fi, float* xb, int lane, int h) {
    constexpr int MT = (N + 15) / 16, KT = N / 8, XS = 2 * N + 4;
    static_assert(QPL * 32 / LPQ == 8, "the tensor-core product wants 8 q per warp");
    static_assert(N % 8 == 0, "the tensor-core product wants whole 8-column tiles");
    __syncwarp();
#pragma unroll
    for (int c = 0; c < QPL; ++c) {
        float* xq = xb + ((lane / LPQ) * QPL + c) * XS;
#pragma unroll
        for (int r = 0; r < RPL; ++r)
            if (h * RPL + r < N) *reinterpret_cast<float2*>(xq + 2 * (h * RPL + r)) = rr[c][r];
    }
    __syncwarp();
    const int g = lane >> 2, t = lane & 3;
    uint32_t bre[KT][2], bim[KT][2], bin[KT][2];
#pragma unroll
    for (int kt = 0; kt < KT; ++kt) {
        const float2 v0 = *reinterpret_cast<const float2*>(xb + g * XS + 2 * (kt * 8 + t));
        const float2 v1 = *reinterpret_cast<const float2*>(xb + g * XS + 2 * (kt * 8 + t + 4));
        bre[kt][0] = to_tf32(v0.x); bre[kt][1] = to_tf32(v1.x);
        bim[kt][0] = to_tf32(v0.y); bim[kt][1] = to_tf32(v1.y);
        bin[kt][0] = to_tf32(-v0.y); bin[kt][1] = to_tf32(-v1.y);
    }
    float dre[MT][4], dim[MT][4];
#pragma unroll
    for (int mt = 0; mt < MT; ++mt) {
#pragma unroll
        for (int e = 0; e < 4; ++e) dre[mt][e] = dim[mt][e] = 0.f;
#pragma unroll
        for (int kt = 0; kt < KT; ++kt) {
            const uint4 ar = fr[(mt * KT + kt) * 32 + lane], ai = fi[(mt * KT + kt) * 32 + lane];
            mma_tf32(dre[mt], ar, bre[kt][0], bre[kt][1]);
            mma_tf32(dre[mt], ai, bin[kt][0], bin[kt][1]);
            mma_tf32(dim[mt], ai, bre[kt][0], bre[kt][1]);
            mma_tf32(dim[mt], ar, bim[kt][0], bim[kt][1]);
        }
    }
    __syncwarp();
#pragma unroll
    for (int mt = 0; mt < MT; ++mt) {
        const int m0 = mt * 16 + g, m1 = m0 + 8;
        if (m0 < N) {
            *reinterpret_cast<float2*>(xb + (2 * t) * XS + 2 * m0) = make_float2(dre[mt][0], dim[mt][0]);
            *reinterpret_cast<float2*>(xb + (2 * t + 1) * XS + 2 * m0) = make_float2(dre[mt][1], dim[mt][1]);
        }
        if (m1 < N) {
            *reinterpret_cast<float2*>(xb + (2 * t) * XS + 2 * m1) = make_float2(dre[mt][2], dim[mt][2]);
            *reinterpret_cast<float2*>(xb + (2 * t + 1) * XS + 2 * m1) = make_float2(dre[mt][3], dim[mt][3]);
        }
    }
    __syncwarp();
#pragma unroll
    for (int c = 0; c < QPL; ++c) {
        const float* xq = xb + ((lane / LPQ) * QPL + c) * XS;
#pragma unroll
        for (int r = 0; r < RPL; ++r)
            dx[c][r] = h * RPL + r < N ? *reinterpret_cast<const float2*>(xq + 2 * (h * RPL + r)) : make_float2(0.f, 0.f);
    }
}

// d += a b, one m8n8k4 FP64 tile (one A and one B fragment value per lane)
__device__ __forceinline__ void mma_f64(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

// acc = B x for the warp's 8 q (the same lane layout as tc_apply) on the FP64 tensor path: gr / gi
// hold the A fragments of Re and Im of the B rows (Gamma^T without the diagonal), tile (mt, kt) at
// [(mt KT + kt) 32 + lane]; xb: this warp's exchange buffer [8 q][XD] doubles, used once for the real
// parts and once for the imaginary parts in each direction.
template <int N, int RPL, int QPL, int LPQ>
__device__ __forceinline__ void dm_apply(const double2 (&x)[QPL][RPL], double2 (&acc)[QPL][RPL], const double* gr,
                                         const double* gi, double* xb, int lane, int h) {
    constexpr int MT = N / 8, KT = N / 4, XD = N + 4;
    static_assert(N % 8 == 0 && QPL * 32 / LPQ == 8, "the FP64 tensor product wants 8-row tiles and 8 q per warp");
    const int g = lane >> 2, t = lane & 3, qb = (lane / LPQ) * QPL;
    double bre[KT], bim[KT];
#pragma unroll
    for (int part = 0; part < 2; ++part) {
        __syncwarp();
#pragma unroll
        for (int c = 0; c < QPL; ++c)
#pragma unroll
            for (int r = 0; r < RPL; ++r)
                if (h * RPL + r < N) xb[(qb + c) * XD + h * RPL + r] = part ? x[c][r].y : x[c][r].x;
        __syncwarp();
#pragma unroll
        for (int kt = 0; kt < KT; ++kt) (part ? bim : bre)[kt] = xb[g * XD + kt * 4 + t];
    }
    double dr[MT][2], di[MT][2];
#pragma unroll
    for (int mt = 0; mt < MT; ++mt) {
        // three real tile products per complex tile (Karatsuba): t1 = Ar xr, t2 = Ai xi,
        // t3 = (Ar + Ai)(xr + xi); Re = t1 - t2, Im = t3 - t1 - t2.  The operand sums are one FP64
        // add per fragment register on the otherwise idle FP64 pipe.
        dr[mt][0] = dr[mt][1] = di[mt][0] = di[mt][1] = 0.0;
        double t2[2] = {0.0, 0.0};
#pragma unroll
        for (int kt = 0; kt < KT; ++kt) {
            const double ar = gr[(mt * KT + kt) * 32 + lane], ai = gi[(mt * KT + kt) * 32 + lane];
            mma_f64(dr[mt], ar, bre[kt]);
            mma_f64(t2, ai, bim[kt]);
            mma_f64(di[mt], ar + ai, bre[kt] + bim[kt]);
        }
        di[mt][0] -= dr[mt][0] + t2[0];
        di[mt][1] -= dr[mt][1] + t2[1];
        dr[mt][0] -= t2[0];
        dr[mt][1] -= t2[1];
    }
#pragma unroll
    for (int part = 0; part < 2; ++part) {
        __syncwarp();
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) {
            xb[(2 * t) * XD + mt * 8 + g] = part ? di[mt][0] : dr[mt][0];
            xb[(2 * t + 1) * XD + mt * 8 + g] = part ? di[mt][1] : dr[mt][1];
        }
        __syncwarp();
#pragma unroll
        for (int c = 0; c < QPL; ++c)
#pragma unroll
            for (int r = 0; r < RPL; ++r)
                if (h * RPL + r < N) {
                    const double v = xb[(qb + c) * XD + h * RPL + r];
                    if (part) acc[c][r].y = v; else acc[c][r].x = v;
                }
    }
}

// perm[w * nq + i]: the i-th q of w in ascending (key, q) order, key = Re 1/chi0(q, nnu/2 - 1, w) +
// Re 1/chi0(q, nnu/2, w) (the two lowest |nu|; on the 3D 32^3 matrices this key gives 8.7 residual
// passes per warp against 9.3 for nnu/2 alone), one CTA per w (nq <= 4096); non-finite keys sort as 0.
// Bitonic sort of P = max(2^ceil(log2 nq), 32) keys (padding +inf) under the total order (key,
// index).  Thread t holds positions t + 1024 r (r < P / 1024) in registers.  A compare-exchange
// whose partner is fewer than 32 positions away stays inside the warp and runs on shuffles; only
// the stages with partner distance >= 32 go through shared memory, each behind one barrier
// (15 of 55 stages at P = 1024).  The sorted order is unique, so any schedule gives the same perm.
constexpr int kQoMaxR = 4;   // P <= 4096
__global__ void __launch_bounds__(1024) k_bse_qorder(int nq, int nnu, const double2* __restrict__ chi0,
                                                     int32_t* __restrict__ perm) {
    extern __shared__ __align__(16) unsigned char qo_raw[];
    int P = 32;
    while (P < nq) P <<= 1;
    const int R = (P + 1023) / 1024;
    double* skey = reinterpret_cast<double*>(qo_raw);
    int* sidx = reinterpret_cast<int*>(skey + P);
    const int w = blockIdx.x, vc = nnu / 2, tid = threadIdx.x;
    double key[kQoMaxR];
    int idx[kQoMaxR];
#pragma unroll
    for (int r = 0; r < kQoMaxR; ++r) {
        const int i = tid + 1024 * r;
        key[r] = INFINITY;
        idx[r] = i;
        if (r < R && i < nq) {
            const double2 z = chi0[(size_t)i + (size_t)nq * (vc + (size_t)nnu * w)];
            const double2 y = chi0[(size_t)i + (size_t)nq * (vc - 1 + (size_t)nnu * w)];
            double k = z.x / (z.x * z.x + z.y * z.y) + y.x / (y.x * y.x + y.y * y.y);
            if (!isfinite(k)) k = 0.0;
            key[r] = k;
        }
    }
    for (int k = 2; k <= P; k <<= 1) {
        int j = k >> 1;
        if (j >= 32) {
            __syncthreads();   // the previous read-back is complete before the buffer is rewritten
#pragma unroll
            for (int r = 0; r < kQoMaxR; ++r) {
                const int i = tid + 1024 * r;
                if (r < R && i < P) { skey[i] = key[r]; sidx[i] = idx[r]; }
            }
            __syncthreads();
            for (; j >= 32; j >>= 1) {
                for (int i = tid; i < P; i += blockDim.x) {
                    const int l = i ^ j;
                    if (l > i) {
                        const bool up = (i & k) == 0;
                        const bool gt = skey[i] > skey[l] || (skey[i] == skey[l] && sidx[i] > sidx[l]);
                        if (gt == up) {
                            const double tk = skey[i]; skey[i] = skey[l]; skey[l] = tk;
                            const int ti = sidx[i]; sidx[i] = sidx[l]; sidx[l] = ti;
                        }
                    }
                }
                __syncthreads();
            }
#pragma unroll
            for (int r = 0; r < kQoMaxR; ++r) {
                const int i = tid + 1024 * r;
                if (r < R && i < P) { key[r] = skey[i]; idx[r] = sidx[i]; }
            }
        }
        for (; j > 0; j >>= 1) {
#pragma unroll
            for (int r = 0; r < kQoMaxR; ++r) {
                if (r < R) {   // uniform over the block: every lane of a warp shuffles together
                    const int i = tid + 1024 * r;
                    const double pk = __shfl_xor_sync(0xffffffffu, key[r], j);
                    const int pi = __shfl_xor_sync(0xffffffffu, idx[r], j);
                    const bool want_min = ((i & k) == 0) == ((i & j) == 0);
                    const bool less = key[r] < pk || (key[r] == pk && idx[r] < pi);
                    if (want_min != less) { key[r] = pk; idx[r] = pi; }
                }
            }
        }
    }
#pragma unroll
    for (int r = 0; r < kQoMaxR; ++r) {
        const int i = tid + 1024 * r;
        if (r < R && i < nq) perm[(size_t)w * nq + i] = idx[r];
    }
}

// identity order (boxes with more than 4096 q)
__global__ void k_bse_qorder_id(int nq, int nw, int32_t* __restrict__ perm) {
    const size_t total = (size_t)nq * nw;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x)
        perm[e] = (int32_t)(e % nq);
}

__device__ __forceinline__ float2 f2_fma(float2 c, float2 r, float2 acc) {
    acc.x = fmaf(c.x, r.x, acc.x);
    acc.x = fmaf(-c.y, r.y, acc.x);
    acc.y = fmaf(c.x, r.y, acc.y);
    acc.y = fmaf(c.y, r.x, acc.y);
    return acc;
}

// NL: the box size Nν of the data; the tiles use N >= NL (a multiple of 8 for the tensor paths).
// Rows and columns NL .. N-1 are an identity block with a zero right-hand side: Gamma^T is padded
// with zeros, 1/chi0 with ones, so x and r stay zero there and the first NL rows solve B y = 1.
template <int N, int LPQ, int QPL, int MINB, bool GSM, bool TC, bool DM, bool P2, bool NS, int NL, bool ADJ = false>
__global__ void __launch_bounds__(kIterQ * LPQ / QPL, MINB) k_bse_iter(const BseArgs a_m, const BseArgs a_d,
                                                                       const int32_t* __restrict__ perm) {
    // blockIdx.z selects the channel: one launch may cover both (they share chi0 and the q order),
    // so the second channel's CTAs fill the SMs the first one's tail leaves idle
    BseArgs a = a_m;
    if (blockIdx.z) {
        a.s = a_d.s; a.Gamma = a_d.Gamma; a.chi = a_d.chi; a.gam = a_d.gam; a.flags = a_d.flags;
        a.fail_list = a_d.fail_list; a.fail_count = a_d.fail_count;
    }
    using S = IterSmem<N, GSM, TC, kIterQ * LPQ / QPL / 32, DM, NS>;
    static_assert(!DM || (GSM && TC), "the FP64 tensor product is built with the tensor-core FP32 product");
    static_assert(!NS || (DM && N % 8 == 0 && kIterQ * LPQ / QPL == 128),
                  "the tensor-core group inverse is built for the DM configuration, 128 threads");
    static_assert(NL <= N && NL % 2 == 0, "padded box");
    static_assert(!ADJ || TC, "general right-hand sides enter through the tensor-core product");
    constexpr int LD = S::LD;
    constexpr int LDG = GSM ? LD : N;   // row stride of Gamma^T where it is read
    constexpr int RPL = (N + LPQ - 1) / LPQ;
    constexpr int NT = kIterQ * LPQ / QPL;
    static_assert(32 % LPQ == 0, "the lanes of one q sit in one warp");
    extern __shared__ __align__(16) unsigned char it_raw[];
    double2* Gs = reinterpret_cast<double2*>(it_raw);
    double2* Dq = reinterpret_cast<double2*>(it_raw + S::off_D);
    float2* C = reinterpret_cast<float2*>(it_raw + S::off_C);
    uint32_t* Cf = reinterpret_cast<uint32_t*>(it_raw + S::off_C);     // TC: [2][MT][KT][32][4] tf32
    float* Xb = reinterpret_cast<float*>(it_raw + S::off_X);           // TC: [warps][8 q][XS]
    double* rowabs = reinterpret_cast<double*>(it_raw + S::off_rowabs);
    double2* dbar = reinterpret_cast<double2*>(it_raw + S::off_dbar);
    float2* pc = reinterpret_cast<float2*>(it_raw + S::off_pc);

    const int tid = threadIdx.x, lane = tid & 31;
    const int w = blockIdx.y, g0 = blockIdx.x * kIterQ;
    const int h = tid % LPQ, gbase = lane - h, ql0 = (tid / LPQ) * QPL;   // this lane group's q: ql0 + c
    const int nvalid = min(kIterQ, a.nq - g0);
    const int32_t* pw = perm + (size_t)w * a.nq + g0;

    // ---- B rows: B_ij = Gamma[w][i N + j] + delta_ij D_i;  D = 1/chi0 of the CTA's q
    // fixed trip counts, fully unrolled: every global load of a thread is in flight at once
    const double2* Gw = a.Gamma + (size_t)w * NL * NL;
    const double2* Gt = GSM ? Gs : Gw;
    // element (i, j) of Gamma(w) as stored, zero in the padding
    auto gglob = [&](int i, int j) -> double2 {
        return (i < NL && j < NL) ? Gw[(size_t)i * NL + j] : dmk(0.0, 0.0);
    };
    double* Gfr = reinterpret_cast<double*>(it_raw);            // DM: A fragments of Re B, then Im B
    double* Gfi = Gfr + N * N;
    // element B_ij without the diagonal term, from wherever Gamma^T is kept
    auto gelt = [&](int i, int j) -> double2 {
        if constexpr (DM) {
            const int f = ((i >> 3) * (N / 4) + (j >> 2)) * 32 + (i & 7) * 4 + (j & 3);
            return dmk(Gfr[f], Gfi[f]);
        } else {
            return Gt[i * LDG + j];
        }
    };
    auto stage_gamma = [&]() {
      if constexpr (GSM) {
        constexpr int NG = (N * N + NT - 1) / NT;
        double2 gv[NG];
#pragma unroll
        for (int m = 0; m < NG; ++m) {
            const int e = tid + NT * m;
            if (e < N * N) gv[m] = NL == N ? Gw[e] : gglob(e / N, e - (e / N) * N);
        }
#pragma unroll
        for (int m = 0; m < NG; ++m) {
            const int e = tid + NT * m;
            if (e < N * N) {
                const int i = e / N, j = e - (e / N) * N;
                if constexpr (DM) {
                    const int f = ((i >> 3) * (N / 4) + (j >> 2)) * 32 + (i & 7) * 4 + (j & 3);
                    Gfr[f] = gv[m].x;
                    Gfi[f] = gv[m].y;
                } else {
                    Gs[i * LD + j] = gv[m];
                }
            }
        }
      }
    };
    // NS: the tensor-core group inverse's mbarrier and TMEM (128 columns; 3 CTAs per SM take 384 of
    // the 512), set up while D loads; Gamma^T is staged after the inverse, whose buffers it reuses
    uint64_t* ns_bar = reinterpret_cast<uint64_t*>(it_raw + S::off_bar);
    uint32_t* ns_slot = reinterpret_cast<uint32_t*>(it_raw + S::off_slot);
    if constexpr (NS) {
        if (tid == 0) {
            tc05::mbar_init(ns_bar, 1);
            tc05::mbar_fence_init();
        }
        if (tid < 32) tc05::tmem_alloc(ns_slot, ns::NsSmem<N>::tmem_cols);
    } else {
        stage_gamma();
    }
    {
        constexpr int ND = (kIterQ * N + NT - 1) / NT;
        int qg[ND];
        double2 cv[ND];
#pragma unroll
        for (int m = 0; m < ND; ++m) {
            const int e = tid + NT * m, qq = e / N;
            qg[m] = (e < kIterQ * N && qq < nvalid) ? pw[qq] : -1;
        }
#pragma unroll
        for (int m = 0; m < ND; ++m) {
            const int e = tid + NT * m, v = e - (e / N) * N;
            // padding rows: chi0 = 1, so D = 1 there
            cv[m] = qg[m] >= 0 ? (v < NL ? a.chi0[(size_t)qg[m] + (size_t)a.nq * (v + (size_t)NL * w)] : dmk(1.0, 0.0))
                               : dmk(0.0, 0.0);
        }
        // 1/chi0 = conj(chi0) / |chi0|^2 by batch inversion (Montgomery's trick): prefix products of
        // the ND squared moduli, one division, two products per reciprocal, instead of ND scaled
        // complex reciprocals (three divisions each) run one after another.  A product outside
        // [1e-300, 1e300] takes cinv element by element.
        double nrm[ND], pre[ND];
        double prod = 1.0;
#pragma unroll
        for (int m = 0; m < ND; ++m) {
            nrm[m] = qg[m] >= 0 ? cv[m].x * cv[m].x + cv[m].y * cv[m].y : 1.0;
            pre[m] = prod;
            prod *= nrm[m];
        }
        if (prod > 1e-300 && prod < 1e300) {
            double r = 1.0 / prod;
#pragma unroll
            for (int m = ND - 1; m >= 0; --m) {
                const double inv = r * pre[m];
                r *= nrm[m];
                const int e = tid + NT * m;
                if (e < kIterQ * N) Dq[e] = qg[m] >= 0 ? dmk(cv[m].x * inv, -cv[m].y * inv) : dmk(0.0, 0.0);
            }
        } else {
#pragma unroll
            for (int m = 0; m < ND; ++m) {
                const int e = tid + NT * m;
                if (e < kIterQ * N) Dq[e] = qg[m] >= 0 ? cinv(cv[m]) : dmk(0.0, 0.0);
            }
        }
    }
    __syncthreads();
    // |row|_1 of Gamma^T (one thread per row) and the group's mean diagonal (one thread per nu, in
    // another warp), each a sequential sum in a fixed order: no shuffle chains on the set-up path
    static_assert(NT >= 64 + N, "row sums in threads 0..N-1, diagonal means in threads 64..63+N");
    auto row_sums = [&]() {
        if (tid < N) {
            double sacc = 0.0;
            for (int j = 0; j < N; ++j) {
                const double2 v = gelt(tid, j);
                sacc += fabs(v.x) + fabs(v.y);
            }
            rowabs[tid] = sacc;
        }
    };
    if constexpr (!NS) row_sums();
    if (tid >= 64 && tid < 64 + N) {
        const int i = tid - 64;
        double2 m = dmk(0.0, 0.0);
        for (int q = 0; q < nvalid; ++q) m = cadd(m, Dq[q * N + i]);
        dbar[i] = cscale(m, 1.0 / (double)max(nvalid, 1));
    }
    __syncthreads();
    // ---- C = B_bar^-1: in-place Gauss-Jordan in FP32 without pivoting (a poor C only costs sweeps),
    // two pivots per step (N is even: N = 2 n_iv).  TPR threads own each row (a contiguous segment of
    // CPT columns each, in registers).  Step k publishes columns k, k+1 and rows k, k+1 to a
    // double-buffered shared block, so one barrier per step suffices (buffer (k/2) & 1 was last read
    // in the step before the previous barrier).  With P the 2 x 2 pivot block, row i outside it takes
    // a_ij -= (a_i,k:k+1 P^-1) . u_k:k+1,j.  The published rows carry P + I in the pivot columns, so
    // the same update writes -(a_i,k:k+1 P^-1) into columns k, k+1 (the Gauss-Jordan column entries)
    // with no per-element branch; the pivot rows become P^-1 u (and P^-1 in the pivot columns, which
    // is the +I term's product minus the identity).  Mathematically two single-pivot steps.
    // elt(i, j): element B_ij without the diagonal term.
    auto gauss_jordan = [&](auto&& elt) {
        static_assert(N % 2 == 0, "pivot pairs");
        constexpr int TPR = NT / N > 0 ? NT / N : 1;
        constexpr int CPT = (N + TPR - 1) / TPR;
        const int gi = tid / TPR, gp = tid - (tid / TPR) * TPR, j0 = gp * CPT;
        const bool own = gi < N;
        float2 ce[CPT];
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
            const int jj = j0 + c;
            ce[c] = make_float2(0.f, 0.f);
            if (own && jj < N) {
                double2 v = elt(gi, jj);
                if (gi == jj) v = cadd(v, dbar[gi]);
                ce[c] = make_float2((float)v.x, (float)v.y);
            }
        }
        static_assert(S::TPR == TPR && S::RW == TPR * CPT, "pivot buffer geometry");
        for (int k = 0; k < N; k += 2) {
            // [N] column k, [N] column k+1, then [RW] (row k, row k+1) pairs; columns >= N of the
            // rows are the owners' zero padding, so the updates below need no column bound
            float2* pb = reinterpret_cast<float2*>(reinterpret_cast<char*>(pc) + ((k >> 1) & 1) * S::pc_half);
            float2* pr = pb + 2 * N;                    // float2 view of the pairs: [2 j + r]
            if (own) {
#pragma unroll
                for (int c = 0; c < CPT; ++c) {
                    const int jj = j0 + c;
                    if (jj == k) pb[gi] = ce[c];
                    if (jj == k + 1) pb[N + gi] = ce[c];
                }
                if (gi == k || gi == k + 1) {
                    const int r = gi - k;
#pragma unroll
                    for (int c = 0; c < CPT; ++c) {
                        const int jj = j0 + c;
                        pr[2 * jj + r] = jj == gi ? make_float2(ce[c].x + 1.f, ce[c].y) : ce[c];
                    }
                }
            }
            __syncthreads();
            if (own) {
                const float4* pq = reinterpret_cast<const float4*>(pr);
                const float2 p00 = pb[k], p10 = pb[k + 1], p01 = pb[N + k], p11 = pb[N + k + 1];
                const float2 pd = fmul(p00, p11), po = fmul(p01, p10);
                const float2 rdet = vinv(make_float2(pd.x - po.x, pd.y - po.y));
                const float2 i00 = fmul(p11, rdet), i11 = fmul(p00, rdet);
                const float2 i01 = fmul(make_float2(-p01.x, -p01.y), rdet);
                const float2 i10 = fmul(make_float2(-p10.x, -p10.y), rdet);
                float2 m0, m1;
                if (gi == k || gi == k + 1) {          // pivot row: P^-1[r, :] u', minus its +1
                    m0 = gi == k ? i00 : i10;
                    m1 = gi == k ? i01 : i11;
#pragma unroll
                    for (int c = 0; c < CPT; ++c) {
                        const int jj = j0 + c;
                        const float4 u = pq[jj];
                        float2 v = fadd(fmul(m0, make_float2(u.x, u.y)), fmul(m1, make_float2(u.z, u.w)));
                        if (jj == gi) v.x -= 1.f;
                        ce[c] = v;
                    }
                } else {                                // m = a_i,k:k+1 P^-1; a_ij -= m . u'_j
                    const float2 a0 = pb[gi], a1 = pb[N + gi];
                    m0 = fadd(fmul(a0, i00), fmul(a1, i10));
                    m1 = fadd(fmul(a0, i01), fmul(a1, i11));
#pragma unroll
                    for (int c = 0; c < CPT; ++c) {
                        const float4 u = pq[j0 + c];
                        float2 v = ce[c];
                        v.x = fmaf(-m0.x, u.x, v.x);
                        v.x = fmaf(m0.y, u.y, v.x);
                        v.y = fmaf(-m0.x, u.y, v.y);
                        v.y = fmaf(-m0.y, u.x, v.y);
                        v.x = fmaf(-m1.x, u.z, v.x);
                        v.x = fmaf(m1.y, u.w, v.x);
                        v.y = fmaf(-m1.x, u.w, v.y);
                        v.y = fmaf(-m1.y, u.z, v.y);
                        ce[c] = v;
                    }
                }
            }
        }
        if constexpr (TC) {
            // A fragments: element (m, k) of a 16 x 8 tile sits in lane 4 (m mod 8) + (k mod 4),
            // register (m / 8) + 2 (k / 4); rows N .. 16 MT - 1 stay zero
            constexpr int FR = S::MT * S::KT * 32 * 4;
            __syncthreads();   // the zeroing below must not overtake the last pivot reads
            for (int e = tid; e < 2 * FR; e += NT) Cf[e] = 0u;
            __syncthreads();
            if (own) {
#pragma unroll
                for (int c = 0; c < CPT; ++c) {
                    const int jj = j0 + c;
                    if (jj < N) {
                        const int mt = gi >> 4, m16 = gi & 15, kt = jj >> 3, k8 = jj & 7;
                        const int idx = ((mt * S::KT + kt) * 32 + (m16 & 7) * 4 + (k8 & 3)) * 4 + (m16 >> 3) + 2 * (k8 >> 2);
                        Cf[idx] = to_tf32(ce[c].x);
                        Cf[FR + idx] = to_tf32(ce[c].y);
                    }
                }
            }
        } else {
            if (own) {
#pragma unroll
                for (int c = 0; c < CPT; ++c)
                    if (j0 + c < N) C[gi * LD + j0 + c] = ce[c];
            }
        }
    };
    if constexpr (!NS) {
        gauss_jordan(gelt);
    } else {
        // ---- C = B_bar^-1 by Newton-Schulz iterations on the tensor cores (ns_inverse.cuh) from the
        // Jacobi seed X_0 = diag(1 / B_bar_ii): B_bar's rows come from Gamma(w) in global memory (L2)
        // and D_bar.  Where the seed is too far (the iteration diverges) the Gauss-Jordan elimination
        // above forms C instead; either way C only sets the sweep count, which the FP64 residual checks.
        using NSm = ns::NsSmem<N>;
        constexpr int FR = S::MT * S::KT * 32 * 4;
        unsigned char* nsb = it_raw;
        float* ns_red = reinterpret_cast<float*>(it_raw + S::off_red);
        // every thread takes elements e = tid + NT m of B_bar (row-major), all loads in flight at
        // once: B_bar_ij into the A buffers, X_0 = diag(1 / B_bar_ii) into the A buffers (row i)
        // and the B buffers (column i; element (j, i))
        {
            constexpr int NE = (N * N + NT - 1) / NT;
            double2 gv[NE];
#pragma unroll
            for (int m = 0; m < NE; ++m) {
                const int e = tid + NT * m;
                gv[m] = e < N * N ? (NL == N ? Gw[e] : gglob(e / N, e - (e / N) * N)) : dmk(0.0, 0.0);
            }
#pragma unroll
            for (int m = 0; m < NE; ++m) {
                const int e = tid + NT * m;
                if (e < N * N) {
                    const int i = e / N, j = e - (e / N) * N;
                    double2 v = gv[m];
                    float2 xv = make_float2(0.f, 0.f);
                    if (i == j) {
                        v = cadd(v, dbar[i]);
                        xv = vinv(make_float2((float)v.x, (float)v.y));
                    }
                    const uint32_t oa = tc05::kmajor_offset(N, i, j), ob = tc05::kmajor_offset(N, j, i);
                    *reinterpret_cast<float*>(nsb + NSm::off_br + oa) = tc05::to_tf32f((float)v.x);
                    *reinterpret_cast<float*>(nsb + NSm::off_bi + oa) = tc05::to_tf32f((float)v.y);
                    *reinterpret_cast<float*>(nsb + NSm::off_xr + oa) = tc05::to_tf32f(xv.x);
                    *reinterpret_cast<float*>(nsb + NSm::off_xi + oa) = tc05::to_tf32f(xv.y);
                    *reinterpret_cast<float*>(nsb + NSm::off_tr + ob) = tc05::to_tf32f(xv.x);
                    *reinterpret_cast<float*>(nsb + NSm::off_ti + ob) = tc05::to_tf32f(xv.y);
                }
            }
        }
        tc05::fence_before();
        __syncthreads();                           // the TMEM address is visible
        tc05::fence_after();
        ns::NsState st{*ns_slot, 0u, true};
        auto emit_cf = [&](int t, int c, const float (&re)[16], const float (&im)[16]) {
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int jj = c + j;
                if (jj < N) {
                    const int mt = t >> 4, m16 = t & 15, kt = jj >> 3, k8 = jj & 7;
                    const int idx = ((mt * S::KT + kt) * 32 + (m16 & 7) * 4 + (k8 & 3)) * 4 + (m16 >> 3) + 2 * (k8 >> 2);
                    Cf[idx] = to_tf32(re[j]);
                    Cf[FR + idx] = to_tf32(im[j]);
                }
            }
        };
        const bool ok = ns::newton_schulz<N>(nsb, ns_bar, ns_red, st, kNsMaxIts, kNsTol, emit_cf, nullptr);
        ns::drain(st, ns_bar);
        tc05::fence_before();
        __syncthreads();
        if (tid < 32) {
            tc05::fence_after();
            tc05::tmem_free(st.tmem, NSm::tmem_cols);
        }
        if (ok) {
            // zero rows N .. 16 MT - 1 of the fragments (the inverse's buffers overlapped them)
            if (tid >= N && tid < 16 * S::MT) {
                for (int jj = 0; jj < N; ++jj) {
                    const int mt = tid >> 4, m16 = tid & 15, kt = jj >> 3, k8 = jj & 7;
                    const int idx = ((mt * S::KT + kt) * 32 + (m16 & 7) * 4 + (k8 & 3)) * 4 + (m16 >> 3) + 2 * (k8 >> 2);
                    Cf[idx] = 0u;
                    Cf[FR + idx] = 0u;
                }
            }
        } else {
            gauss_jordan(gglob);
        }
        __syncthreads();
        stage_gamma();
        __syncthreads();
        row_sums();
    }
    __syncthreads();

    // ---- per q: norm of B_q's rows, x = C 1 (ADJ: x = C b, b and max |b| in registers)
    double rown[QPL];
    double2 x[QPL][RPL];
    double2 bq[ADJ ? QPL : 1][ADJ ? RPL : 1];
    double bn[ADJ ? QPL : 1];
#pragma unroll
    for (int c = 0; c < QPL; ++c) rown[c] = 0.0;
#pragma unroll
    for (int c = 0; c < (ADJ ? QPL : 1); ++c) bn[c] = 0.0;
#pragma unroll
    for (int r = 0; r < RPL; ++r) {
        const int i = h * RPL + r;
        float2 sacc = make_float2(0.f, 0.f);
        double rowg = 0.0;
        double2 g = dmk(0.0, 0.0);
        if (N % LPQ == 0 || i < N) {
            g = gelt(i, i);
            rowg = rowabs[i] - (fabs(g.x) + fabs(g.y));
            if constexpr (!TC) {
                float2 s2 = make_float2(0.f, 0.f);
#pragma unroll
                for (int j = 0; j < NL; j += 2) {          // C 1 over the box's columns
                    sacc = fadd(sacc, C[i * LD + j]);
                    if (j + 1 < NL) s2 = fadd(s2, C[i * LD + j + 1]);
                }
                sacc = fadd(sacc, s2);
            }
        }
#pragma unroll
        for (int c = 0; c < QPL; ++c) {
            x[c][r] = dmk(0.0, 0.0);
            if (N % LPQ == 0 || i < N) {
                const double2 d = Dq[(ql0 + c) * N + i];
                rown[c] = fmax(rown[c], rowg + fabs(g.x + d.x) + fabs(g.y + d.y));
                x[c][r] = dmk((double)sacc.x, (double)sacc.y);
            }
            if constexpr (ADJ) {
                double2& b = bq[ADJ ? c : 0][ADJ ? r : 0];
                b = dmk(0.0, 0.0);
                if (i < NL && ql0 + c < nvalid) b = a.rhs[(size_t)pw[ql0 + c] + (size_t)a.nq * (i + (size_t)NL * w)];
                bn[ADJ ? c : 0] = fmax(bn[ADJ ? c : 0], fabs(b.x) + fabs(b.y));
            }
        }
    }
    const uint4* Ffr = reinterpret_cast<const uint4*>(Cf);
    const uint4* Ffi = Ffr + S::MT * S::KT * 32;
    float* xbw = reinterpret_cast<float*>(reinterpret_cast<char*>(Xb) + (tid >> 5) * S::xw_bytes);
    // P2: the correction C r becomes C r - C (ΔD_q ⊙ C r), ΔD_q = D_q - D_bar: the first two terms of
    // (B_bar + ΔD_q)^-1 = (I + C ΔD_q)^-1 C, so one sweep contracts the error by (C ΔD_q)^2 instead of
    // C ΔD_q.  The extra product is a second TF32 tensor-core product, cheap beside the FP64 residual:
    // on the 3D 32^3 matrices the residual passes per warp fall from 8.6 to 5.1.  z = ΔD ⊙ v in FP32.
    auto second_order = [&](float2 (&v)[QPL][RPL], float2 (&z)[QPL][RPL]) {
      if constexpr (TC && P2) {
#pragma unroll
        for (int c = 0; c < QPL; ++c)
#pragma unroll
            for (int r = 0; r < RPL; ++r) {
                const int i = h * RPL + r;
                z[c][r] = make_float2(0.f, 0.f);
                if (N % LPQ == 0 || i < N) {
                    const double2 d = Dq[(ql0 + c) * N + i], db = dbar[i];
                    z[c][r] = fmul(make_float2((float)(d.x - db.x), (float)(d.y - db.y)), v[c][r]);
                }
            }
        tc_apply<N, RPL, QPL, LPQ>(z, z, Ffr, Ffi, xbw, lane, h);   // inputs are staged before outputs land
#pragma unroll
        for (int c = 0; c < QPL; ++c)
#pragma unroll
            for (int r = 0; r < RPL; ++r) v[c][r] = make_float2(v[c][r].x - z[c][r].x, v[c][r].y - z[c][r].y);
      }
    };
    if constexpr (TC) {   // x = C 1 through the same tensor-core product
        float2 one[QPL][RPL], d0[QPL][RPL];
#pragma unroll
        for (int c = 0; c < QPL; ++c)
#pragma unroll
            for (int r = 0; r < RPL; ++r)
                one[c][r] = ADJ ? make_float2((float)bq[ADJ ? c : 0][ADJ ? r : 0].x, (float)bq[ADJ ? c : 0][ADJ ? r : 0].y)
                                : make_float2(h * RPL + r < NL ? 1.f : 0.f, 0.f);
        tc_apply<N, RPL, QPL, LPQ>(one, d0, Ffr, Ffi, xbw, lane, h);
        if constexpr (P2) second_order(d0, one);
#pragma unroll
        for (int c = 0; c < QPL; ++c)
#pragma unroll
            for (int r = 0; r < RPL; ++r)
                if (N % LPQ == 0 || h * RPL + r < N) x[c][r] = dmk((double)d0[c][r].x, (double)d0[c][r].y);
    }
    bool conv[QPL];
    double berr[QPL];
#pragma unroll
    for (int c = 0; c < QPL; ++c) {
#pragma unroll
        for (int o = 1; o < LPQ; o <<= 1) {
            rown[c] = fmax(rown[c], __shfl_xor_sync(0xffffffffu, rown[c], o));
            if constexpr (ADJ) bn[ADJ ? c : 0] = fmax(bn[ADJ ? c : 0], __shfl_xor_sync(0xffffffffu, bn[ADJ ? c : 0], o));
        }
        conv[c] = ql0 + c >= nvalid;
        berr[c] = 0.0;
    }

    int passes = 0;
    for (int it = 0;; ++it) {
        // residual r = 1 - B_q x (FP64); the source-lane loop stays rolled (code size); every Gamma^T
        // element read from shared memory serves the QPL q of the lane group
        double2 acc[QPL][RPL];
#pragma unroll
        for (int c = 0; c < QPL; ++c)
#pragma unroll
            for (int r = 0; r < RPL; ++r) acc[c][r] = dmk(0.0, 0.0);
        if constexpr (DM) {
            dm_apply<N, RPL, QPL, LPQ>(x, acc, Gfr, Gfi, reinterpret_cast<double*>(xbw), lane, h);
        } else {
#pragma unroll 1
        for (int s = 0; s < LPQ; ++s) {
            const double2* grow = Gt + (size_t)(h * RPL) * LDG + s * RPL;
#pragma unroll
            for (int j = 0; j < RPL; ++j) {
                double2 xk[QPL];
#pragma unroll
                for (int c = 0; c < QPL; ++c) xk[c] = shfl_v(x[c][j], gbase + s);
                if (N % LPQ != 0 && s * RPL + j >= N) continue;
#pragma unroll
                for (int r = 0; r < RPL; ++r) {
                    if (N % LPQ == 0 || h * RPL + r < N) {
                        const double2 g = grow[r * LDG + j];
#pragma unroll
                        for (int c = 0; c < QPL; ++c) {
                            acc[c][r].x = fma(g.x, xk[c].x, acc[c][r].x);
                            acc[c][r].x = fma(-g.y, xk[c].y, acc[c][r].x);
                            acc[c][r].y = fma(g.x, xk[c].y, acc[c][r].y);
                            acc[c][r].y = fma(g.y, xk[c].x, acc[c][r].y);
                        }
                    }
                }
            }
        }
        }
        float2 rr[QPL][RPL];
        bool all = true;
#pragma unroll
        for (int c = 0; c < QPL; ++c) {
            double res = 0.0, xn = 0.0;
#pragma unroll
            for (int r = 0; r < RPL; ++r) {
                const int i = h * RPL + r;
                rr[c][r] = make_float2(0.f, 0.f);
                if (N % LPQ == 0 || i < N) {
                    const double2 t = cadd(acc[c][r], cmul(Dq[(ql0 + c) * N + i], x[c][r]));
                    const double2 bv = ADJ ? bq[ADJ ? c : 0][ADJ ? r : 0] : dmk(i < NL ? 1.0 : 0.0, 0.0);
                    const double rx = bv.x - t.x, ry = bv.y - t.y;
                    res = fmax(res, fabs(rx) + fabs(ry));
                    xn = fmax(xn, fabs(x[c][r].x) + fabs(x[c][r].y));
                    rr[c][r] = make_float2((float)rx, (float)ry);
                }
            }
#pragma unroll
            for (int o = 1; o < LPQ; o <<= 1) {
                res = fmax(res, __shfl_xor_sync(0xffffffffu, res, o));
                xn = fmax(xn, __shfl_xor_sync(0xffffffffu, xn, o));
            }
            // normwise backward error |b - B x| / (|B| |x| + |b|), |b| = 1 for the forward solve
            if (!conv[c]) berr[c] = res / (rown[c] * xn + (ADJ ? bn[ADJ ? c : 0] : 1.0));
            conv[c] = conv[c] || berr[c] <= kIterTol;
            all = all && conv[c];
        }
        passes = it + 1;
        if (__all_sync(0xffffffffu, all) || it >= a.max_sweeps) break;
        // correction x += C r (FP32 product; every C element read serves the QPL q)
        float2 dx[QPL][RPL];
        if constexpr (TC) {
            tc_apply<N, RPL, QPL, LPQ>(rr, dx, Ffr, Ffi, xbw, lane, h);
            if constexpr (P2) second_order(dx, rr);   // rr is free after the first product
        } else {
#pragma unroll
        for (int c = 0; c < QPL; ++c)
#pragma unroll
            for (int r = 0; r < RPL; ++r) dx[c][r] = make_float2(0.f, 0.f);
#pragma unroll 1
        for (int s = 0; s < LPQ; ++s) {
            const float2* crow = C + (size_t)(h * RPL) * LD + s * RPL;
#pragma unroll
            for (int j = 0; j < RPL; ++j) {
                float2 rk[QPL];
#pragma unroll
                for (int c = 0; c < QPL; ++c) rk[c] = shfl_v(rr[c][j], gbase + s);
                if (N % LPQ != 0 && s * RPL + j >= N) continue;
#pragma unroll
                for (int r = 0; r < RPL; ++r)
                    if (N % LPQ == 0 || h * RPL + r < N) {
                        const float2 cv = crow[r * LD + j];
#pragma unroll
                        for (int c = 0; c < QPL; ++c) dx[c][r] = f2_fma(cv, rk[c], dx[c][r]);
                    }
            }
        }
        }
#pragma unroll
        for (int c = 0; c < QPL; ++c)
            if (!conv[c]) {
#pragma unroll
                for (int r = 0; r < RPL; ++r) {
                    x[c][r].x += (double)dx[c][r].x;
                    x[c][r].y += (double)dx[c][r].y;
                }
            }
    }

    if (a.stats && lane == 0) {
        atomicAdd(&a.stats[0], (unsigned long long)passes);
        atomicAdd(&a.stats[1], 1ull);
    }

    // ---- chi, gamma = x / (chi0 (1 + s U chi)), flag.  A q that did not reach kIterTol goes to the
    // pivoted solve: between 1e-14 and the LU kernels' 1e-12 the forward error (condition number x
    // backward error) could exceed the FP64 target.
#pragma unroll
    for (int c = 0; c < QPL; ++c) {
        double sx = 0.0;
#pragma unroll
        for (int r = 0; r < RPL; ++r)
            if (h * RPL + r < NL) sx += x[c][r].x;
#pragma unroll
        for (int o = 1; o < LPQ; o <<= 1) sx += __shfl_xor_sync(0xffffffffu, sx, o);
        const int ql = ql0 + c;
        if (ql >= nvalid) continue;
        const int q = pw[ql];
        const double chi = sx / (a.beta * a.beta);
        const bool ok = isfinite(berr[c]) && berr[c] <= kIterTol;
        if constexpr (ADJ) {          // the adjoint's z = conj(x) and the flag; no chi, no gamma
            if (h == 0) {
                a.flags[(size_t)q + (size_t)a.nq * w] = ok ? 0 : 1;
                if (!ok && a.fail_list) a.fail_list[atomicAdd(a.fail_count, 1)] = q + a.nq * w;
            }
#pragma unroll
            for (int r = 0; r < RPL; ++r) {
                const int i = h * RPL + r;
                if (i < NL) a.gam[(size_t)q + (size_t)a.nq * (i + (size_t)NL * w)] = cconj(x[c][r]);
            }
            continue;
        }
        if (h == 0) {
            a.chi[(size_t)q + (size_t)a.nq * w] = chi;
            a.flags[(size_t)q + (size_t)a.nq * w] = ok ? 0 : 1;
            if (!ok && a.fail_list) a.fail_list[atomicAdd(a.fail_count, 1)] = q + a.nq * w;
        }
        const double rf = 1.0 / (1.0 + a.s * a.U * chi);
#pragma unroll
        for (int r = 0; r < RPL; ++r) {
            const int i = h * RPL + r;
            if (i < NL)
                a.gam[(size_t)q + (size_t)a.nq * (i + (size_t)NL * w)] = cscale(cmul(x[c][r], Dq[ql * N + i]), rf);
        }
    }
}

// ------------------------------------------------------------------------------------------------
// Adjoint (vector-Jacobian product) of the BSE step.  For a real loss L with upstream gradients
// chi_bar (real) and gamma_bar (complex, dL/dRe + i dL/dIm) per (q, w):
//   forward: B = Gamma(w)^T + diag(d), d = 1/chi0, y = B^-1 1, chi = Re sum y / beta^2,
//            gamma = y d rf, rf = 1/(1 + s U chi)
//   y from the forward outputs: y = gamma chi0 / rf (no forward solve is repeated)
//   chi_bar_tot = chi_bar - s U rf^2 sum_i Re(conj(gamma_bar_i) y_i d_i)
//   y_bar_i = conj(d_i rf) gamma_bar_i + chi_bar_tot / beta^2
//   z = B^-H y_bar  <=>  (Gamma(w) + diag(d)) conj(z) = conj(y_bar): the same LU kernel on the
//       untransposed vertex (one FP64 solve per matrix, verified by its backward error)
//   B_bar = -z y^H  ->  Gamma_bar(w)[a, b] = -sum_q conj(y_a) z_b  (k_bse_gamma_grad)
//   chi0_bar_i = -conj(d_i^2) (conj(y_i rf) gamma_bar_i - z_i conj(y_i))
// This is the chi-bar contraction of the inverse, chi^T chi_bar chi^T, restricted to the single
// right-hand side the forward pass used.
struct BseAdjArgs {
    int nq, nnu, nw, qchunk;
    double beta, U;
    int s;
    const double2* Gamma;     // [N, N, Nw]
    const double2* chi0;      // [Nq, N, Nw]
    const double* chi;        // [Nq, Nw]      forward chi_r
    const double2* gam;       // [Nq, N, Nw]   forward gamma_r
    const double* chi_bar;    // [Nq, Nw]      (may be null: zero)
    const double2* gam_bar;   // [Nq, N, Nw]   (may be null: zero)
    double2* chi0_bar;        // [Nq, N, Nw]   out (added to when accumulate)
    int accumulate;
    double2* ybuf;            // [Nq, N, Nw]   out: y
    double2* zbuf;            // [Nq, N, Nw]   out: z
    int32_t* flags;           // [Nq, Nw]      1: backward error above 1e-12
    const int32_t* list = nullptr;    // k_bse_adj: only these (q + Nq w), count[0] of them
    const int32_t* count = nullptr;
};

template <int N, int T, int MINB>
__global__ void __launch_bounds__(T * T, MINB) k_bse_adj(const BseAdjArgs a) {
    using LS = LuSmem<N, T>;
    constexpr int RT = LS::RT, G = LS::G;
    constexpr int CT = (N + 1 + T - 1) / T;
    constexpr int TCN = N % T, CN = N / T;
    static_assert(T <= 32 && 32 % T == 0, "a row group must sit inside one warp");
    extern __shared__ double2 sm[];
    double2* Gsm = sm;                                    // Gamma[j + N*i] at i*N + j
    const int t = threadIdx.x;
    const int tr = t / T, tc = t - (t / T) * T;
    const int lane = t & 31;
    const int bar = 1;
    double2* rowbuf = Gsm + N * N;                        // [2][RW]
    double2* colbuf = rowbuf + 2 * LS::RW;                // [2][CW]
    double2* pinv = colbuf + 2 * LS::CW;                  // [N]
    double2* dinv = pinv + N;                             // [N]
    double2* xsm = dinv + N;                              // [N] solution of (Gamma + D) x = rhs
    double* red = reinterpret_cast<double*>(xsm + N);     // [8 * G/32]
    double2* rhs = reinterpret_cast<double2*>(red + 8 * (G / 32) + 2);   // [N] conj(y_bar)
    double2* yfw = rhs + N;                               // [N] forward y

    auto stage = [&](int w) {
        const double2* Gw = a.Gamma + (size_t)w * N * N;
        for (int e = t; e < N * N; e += blockDim.x) Gsm[e] = Gw[e];
        __syncthreads();
    };
    const unsigned gmask = (T == 32 ? 0xffffffffu : ((1u << T) - 1u)) << (lane & ~(T - 1));

    // one (q, w) with Gamma(w) staged; every thread of the CTA calls it
    auto solve = [&](int q, int w) {
        const size_t cq = (size_t)q + (size_t)a.nq * w;
        const double chi = a.chi[cq];
        const double f = 1.0 + a.s * a.U * chi, rf = 1.0 / f;
        // ---- y from the forward outputs, and y_bar
        double s1 = 0.0;
        for (int i = t; i < N; i += G) {
            const size_t ci = (size_t)q + (size_t)a.nq * (i + (size_t)N * w);
            const double2 c0 = a.chi0[ci];
            const double2 d = cinv(c0);
            const double2 y = cscale(cmul(a.gam[ci], c0), f);
            dinv[i] = d;
            yfw[i] = y;
            if (a.gam_bar) {
                const double2 gb = a.gam_bar[ci], yd = cmul(y, d);
                s1 += gb.x * yd.x + gb.y * yd.y;   // Re(conj(gb) y d)
            }
        }
        {
            double v[1] = {s1};
            const int op[1] = {0};
            group_reduce<1, G>(v, op, red, bar, t);   // its barriers also publish dinv / yfw
            s1 = v[0];
        }
        const double xbar = (a.chi_bar ? a.chi_bar[cq] : 0.0) - a.s * a.U * rf * rf * s1;
        for (int i = t; i < N; i += G) {
            const size_t ci = (size_t)q + (size_t)a.nq * (i + (size_t)N * w);
            double2 yb = make_double2(xbar / (a.beta * a.beta), 0.0);
            if (a.gam_bar) yb = cadd(yb, cmul(cconj(cscale(dinv[i], rf)), a.gam_bar[ci]));
            rhs[i] = cconj(yb);
        }
        named_barrier(bar, G);
        // ---- tile of [A | conj(y_bar)], A_ij = Gamma[i, j] + delta_ij d_i (the untransposed vertex)
        double2 b[RT][CT];
#pragma unroll
        for (int ra = 0; ra < RT; ++ra) {
            const int i = tr + T * ra;
#pragma unroll
            for (int c = 0; c < CT; ++c) {
                const int j = tc + T * c;
                double2 v = dmk(0.0, 0.0);
                if (i < N) {
                    if (j < N) {
                        v = Gsm[j * N + i];
                        if (c == ra && tr == tc) v = cadd(v, dinv[i]);
                    } else if (j == N) {
                        v = rhs[i];
                    }
                }
                b[ra][c] = v;
            }
        }
        // ---- forward elimination and block back substitution (as k_bse_lu)
#pragma unroll
        for (int kc = 0; kc < RT; ++kc) {
            const int kend = (N - T * kc) < T ? (N - T * kc) : T;
#pragma unroll 1
            for (int ktc = 0; ktc < kend; ++ktc) {
                const int k = ktc + T * kc;
                double2* rb = rowbuf + (k & 1) * LS::RW;
                double2* cb = colbuf + (k & 1) * LS::CW;
                if (tr == ktc) {
                    double2 p;
                    p.x = __shfl_sync(gmask, b[kc][kc].x, ktc, T);
                    p.y = __shfl_sync(gmask, b[kc][kc].y, ktc, T);
                    const double2 inv = vinv(p);
                    if (tc == ktc) pinv[k] = inv;
#pragma unroll
                    for (int c = kc; c < CT; ++c) rb[tc + T * c] = vmul<double2>(b[kc][c], inv);
                }
                if (tc == ktc) {
#pragma unroll
                    for (int ra = kc; ra < RT; ++ra) cb[tr + T * ra] = b[ra][kc];
                }
                named_barrier(bar, G);
                double2 u[CT];
#pragma unroll
                for (int c = kc; c < CT; ++c) u[c] = rb[tc + T * c];
#pragma unroll
                for (int ra = kc; ra < RT; ++ra) {
                    if (ra > kc || tr != ktc) {
                        const double2 m = cb[tr + T * ra];
#pragma unroll
                        for (int c = kc; c < CT; ++c) {
                            if (c > kc || tc > ktc) vfnms<double2>(b[ra][c], m, u[c]);
                        }
                    }
                }
            }
        }
        double2 acc[RT];
#pragma unroll
        for (int ra = 0; ra < RT; ++ra) acc[ra] = dmk(0.0, 0.0);
#pragma unroll
        for (int r = RT - 1; r >= 0; --r) {
            const int nb = (N - T * r) < T ? (N - T * r) : T;
            double2 sv = acc[r];
#pragma unroll
            for (int o = 1; o < T; o <<= 1) {
                sv.x += __shfl_xor_sync(0xffffffffu, sv.x, o);
                sv.y += __shfl_xor_sync(0xffffffffu, sv.y, o);
            }
            if (tc == TCN && tr < nb) xsm[T * r + tr] = cmul(csub(b[r][CN], sv), pinv[T * r + tr]);
            named_barrier(bar, G);
            if (r > 0 && T * r + tc < N) {
                const double2 xj = xsm[T * r + tc];
#pragma unroll
                for (int ra = 0; ra < r; ++ra) acc[ra] = cadd(acc[ra], cmul(b[ra][r], xj));
            }
        }
        // ---- FP64 backward error |rhs - A x| / (|A| |x| + |rhs|)
        double st[4] = {0.0, 0.0, 0.0, 0.0};
        const int op[4] = {1, 1, 1, 1};
#pragma unroll
        for (int ra = 0; ra < RT; ++ra) {
            const int i = tr + T * ra;
            double2 accr = dmk(0.0, 0.0);
            double rown = 0.0;
            if (i < N) {
#pragma unroll
                for (int c = 0; c < CT; ++c) {
                    const int j = tc + T * c;
                    if (j < N) {
                        double2 gv = Gsm[j * N + i];
                        if (c == ra && tr == tc) gv = cadd(gv, dinv[i]);
                        accr = cadd(accr, cmul(gv, xsm[j]));
                        rown += fabs(gv.x) + fabs(gv.y);
                    }
                }
            }
#pragma unroll
            for (int o = 1; o < T; o <<= 1) {
                accr.x += __shfl_xor_sync(0xffffffffu, accr.x, o);
                accr.y += __shfl_xor_sync(0xffffffffu, accr.y, o);
                rown += __shfl_xor_sync(0xffffffffu, rown, o);
            }
            if (i < N && tc == 0) {
                const double2 r = csub(rhs[i], accr), xv = xsm[i];
                st[0] = fmax(st[0], fabs(r.x) + fabs(r.y));
                st[1] = fmax(st[1], fabs(xv.x) + fabs(xv.y));
                st[2] = fmax(st[2], rown);
                st[3] = fmax(st[3], fabs(rhs[i].x) + fabs(rhs[i].y));
            }
        }
        group_reduce<4, G>(st, op, red, bar, t);
        const double berr = st[0] / (st[2] * st[1] + st[3] + 1e-300);
        if (t == 0) a.flags[cq] = (isfinite(berr) && berr <= 1e-12) ? 0 : 1;
        // ---- z = conj(x); chi0_bar; y and z for the vertex gradient
        for (int i = t; i < N; i += G) {
            const size_t ci = (size_t)q + (size_t)a.nq * (i + (size_t)N * w);
            const double2 z = cconj(xsm[i]), y = yfw[i], d = dinv[i];
            double2 db = cscale(cmul(z, cconj(y)), -1.0);                        // from B
            if (a.gam_bar) db = cadd(db, cmul(cconj(cscale(y, rf)), a.gam_bar[ci]));   // from gamma
            const double2 c0b = cscale(cmul(cconj(cmul(d, d)), db), -1.0);
            a.chi0_bar[ci] = a.accumulate ? cadd(a.chi0_bar[ci], c0b) : c0b;
            a.ybuf[ci] = y;
            a.zbuf[ci] = z;
        }
        named_barrier(bar, G);
    };
    if (a.list) {
        // the matrices a preconditioned adjoint solve left above its bound, q + Nq w each
        const int n = min(max(a.count[0], 0), a.nq * a.nw);
        for (int item = blockIdx.x; item < n; item += gridDim.x) {
            const int lin = a.list[item];
            stage(lin / a.nq);
            solve(lin % a.nq, lin / a.nq);
        }
        return;
    }
    const int q0 = blockIdx.x * a.qchunk;
    const int q1 = min(a.nq, q0 + a.qchunk);
    stage(blockIdx.y);
    for (int q = q0; q < q1; ++q) solve(q, blockIdx.y);
}

// Gamma_bar(w)[a, b] = -sum_q conj(y[q, a, w]) z[q, b, w], one CTA per (w, 32 x 32 output tile);
// q is staged through shared memory in chunks, summed in a fixed order.
__global__ void __launch_bounds__(256) k_bse_gamma_grad(int nq, int n, const double2* __restrict__ y,
                                                        const double2* __restrict__ z, double2* __restrict__ gbar) {
    constexpr int TQ = 16;
    __shared__ double2 ys[TQ][32], zs[TQ][32];
    const int w = blockIdx.z;
    const int a0 = blockIdx.x * 32, b0 = blockIdx.y * 32;
    const int ta = threadIdx.x & 31, tb = threadIdx.x >> 5;   // 32 x 8 threads, 4 outputs each
    double2 acc[4] = {dmk(0, 0), dmk(0, 0), dmk(0, 0), dmk(0, 0)};
    for (int qc = 0; qc < nq; qc += TQ) {
        for (int e = threadIdx.x; e < TQ * 32; e += blockDim.x) {
            const int qq = e / 32, jj = e % 32;
            const int qi = qc + qq;
            const bool ok = qi < nq;
            ys[qq][jj] = (ok && a0 + jj < n) ? y[(size_t)qi + (size_t)nq * (a0 + jj + (size_t)n * w)] : dmk(0, 0);
            zs[qq][jj] = (ok && b0 + jj < n) ? z[(size_t)qi + (size_t)nq * (b0 + jj + (size_t)n * w)] : dmk(0, 0);
        }
        __syncthreads();
#pragma unroll
        for (int qq = 0; qq < TQ; ++qq) {
            const double2 ya = cconj(ys[qq][ta]);
#pragma unroll
            for (int r = 0; r < 4; ++r) acc[r] = cadd(acc[r], cmul(ya, zs[qq][tb + 8 * r]));
        }
        __syncthreads();
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int aa = a0 + ta, bb = b0 + tb + 8 * r;
        if (aa < n && bb < n) gbar[(size_t)aa + (size_t)n * (bb + (size_t)n * w)] = cscale(acc[r], -1.0);
    }
}

template <int N, int T, int MINB>
int run_bse_adj(ldga_ctx* ctx, const BseAdjArgs& a0) {
    BseAdjArgs a = a0;
    const size_t sm = (size_t)N * N * sizeof(double2) + LuSmem<N, T>::bytes + 2 * N * sizeof(double2) + 16;
    auto kern = k_bse_adj<N, T, MINB>;
    LDGA_CUDA(ctx, set_smem(ctx, kern, sm));
    int chunk = 4;
    while (chunk > 1 && (long)((a.nq + chunk - 1) / chunk) * a.nw < 8 * 148) --chunk;
    a.qchunk = chunk;
    dim3 grid((a.nq + chunk - 1) / chunk, a.nw);
    kern<<<grid, T * T, sm, ctx->stream>>>(a);
    LDGA_LAUNCHED(ctx, "k_bse_adj");
    return LDGA_OK;
}

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

// Fallback: partial-pivoting FP64 LU of B = A^T (one matrix per CTA, shared memory), used for flagged
// matrices and for box sizes without a tiled instantiation.  list == nullptr: all (q, w);
// count_dev (may be null) holds the number of list entries (written earlier on the stream).
// gscratch (may be null): LDGA_PIVOT_GRID matrices in HBM, used when [N][N+1] exceeds shared memory.
// One flagged matrix lin = q + Nq w: the pivoted FP64 LU of [B | 1] in B (the CTA's [N][N+1] scratch);
// writes chi, gamma and the flag (0 solved, 2 non-finite); returns true when chi is finite.  Every
// thread of the CTA calls it.
__device__ bool pivot_solve(const BseArgs& a, int lin, double2* B, double* red, int* piv_s) {
    const int N = a.nnu;
    const int ld = N + 1;
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
    return isfinite(chi);
}

__global__ void __launch_bounds__(256) k_bse_lu_pivot(const BseArgs a, const int32_t* list, int count,
                                                       const int32_t* count_dev, double2* gscratch) {
    extern __shared__ double2 sm[];
    const int N = a.nnu;
    double* red = reinterpret_cast<double*>(sm);                      // [64]
    int* piv_s = reinterpret_cast<int*>(red + 64);                    // [4]
    double2* B = gscratch ? gscratch + (size_t)blockIdx.x * N * (N + 1)   // [N][N+1] row-major, rhs last
                          : reinterpret_cast<double2*>(piv_s + 4);
    if (count_dev) count = count_dev[0];
    for (int item = blockIdx.x; item < count; item += gridDim.x) pivot_solve(a, list ? list[item] : item, B, red, piv_s);
}

// Both channels' flagged matrices of a two-channel preconditioned solve in one launch: the lists the
// solve appended (counts on the device), items of m first; a matrix whose result stays non-finite
// adds one to *d_fail.
__global__ void __launch_bounds__(256) k_bse_lu_pivot_pair(const BseArgs am, const BseArgs ad, double2* gscratch,
                                                            int32_t* d_fail) {
    extern __shared__ double2 sm[];
    const int N = am.nnu;
    double* red = reinterpret_cast<double*>(sm);
    int* piv_s = reinterpret_cast<int*>(red + 64);
    double2* B = gscratch ? gscratch + (size_t)blockIdx.x * N * (N + 1) : reinterpret_cast<double2*>(piv_s + 4);
    // the lists hold at most one entry per (q, w) of the launch
    const int cap = am.nq * am.nw;
    const int cm = min(max(am.fail_count[0], 0), cap), cd = min(max(ad.fail_count[0], 0), cap);
    for (int item = blockIdx.x; item < cm + cd; item += gridDim.x) {
        const bool is_m = item < cm;
        const bool ok = is_m ? pivot_solve(am, am.fail_list[item], B, red, piv_s)
                             : pivot_solve(ad, ad.fail_list[item - cm], B, red, piv_s);
        if (threadIdx.x == 0 && !ok) atomicAdd(d_fail, 1);
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

template <int N, int TR, int TC, int MPC, int MINB, typename TF, int MODE>
int run_tile(ldga_ctx* ctx, const BseArgs& a0) {
    BseArgs a = a0;
    using V = typename C2<TF>::T;
    const int threads = TR * TC * MPC;
    const size_t sm = (size_t)N * N * sizeof(double2) + MPC * group_smem<N, TR, TC, V>();
    auto kern = k_bse_tile<N, TR, TC, MPC, MINB, TF, MODE>;
    LDGA_CUDA(ctx, set_smem(ctx, kern, sm));
    // q chunk: every group of the CTA takes several q of the same w (Gamma(w) staged once)
    int chunk = 4 * MPC;
    while (chunk > MPC && (long)((a.nq + chunk - 1) / chunk) * a.nw < 8 * 148) chunk -= MPC;
    a.qchunk = chunk;
    dim3 grid((a.nq + chunk - 1) / chunk, a.nw);
    StageTimer st_(ctx, LDGA_STAGE_BSE);
    kern<<<grid, threads, sm, ctx->stream>>>(a);
    LDGA_LAUNCHED(ctx, "k_bse_tile");
    return LDGA_OK;
}

template <int N, int T, int MPC, int MINB, bool GSM = true, bool LA = LDGA_LU_LOOKAHEAD>
int run_lu(ldga_ctx* ctx, const BseArgs& a0) {
    BseArgs a = a0;
    const int threads = T * T * MPC;
    const size_t sm = (GSM ? (size_t)N * N * sizeof(double2) : 0) + MPC * LuSmem<N, T>::bytes;
    auto kern = k_bse_lu<N, T, MPC, MINB, GSM, LA>;
    LDGA_CUDA(ctx, set_smem(ctx, kern, sm));
    int chunk = 4 * MPC;
    while (chunk > MPC && (long)((a.nq + chunk - 1) / chunk) * a.nw < 8 * 148) chunk -= MPC;
    a.qchunk = chunk;
    dim3 grid((a.nq + chunk - 1) / chunk, a.nw);
    StageTimer st_(ctx, LDGA_STAGE_BSE);
    kern<<<grid, threads, sm, ctx->stream>>>(a);
    LDGA_LAUNCHED(ctx, "k_bse_lu");
    return LDGA_OK;
}

template <int N, int T, int MPC, int MINB, bool GSM = true>
int run_lu32(ldga_ctx* ctx, const BseArgs& a0) {
    BseArgs a = a0;
    const int threads = T * T * MPC;
    const size_t sm = (GSM ? (size_t)N * N * sizeof(double2) : 0) + MPC * Lu32Smem<N, T>::bytes;
    auto kern = k_bse_lu32<N, T, MPC, MINB, GSM>;
    LDGA_CUDA(ctx, set_smem(ctx, kern, sm));
    int chunk = 4 * MPC;
    while (chunk > MPC && (long)((a.nq + chunk - 1) / chunk) * a.nw < 8 * 148) chunk -= MPC;
    a.qchunk = chunk;
    dim3 grid((a.nq + chunk - 1) / chunk, a.nw);
    StageTimer st_(ctx, LDGA_STAGE_BSE);
    kern<<<grid, threads, sm, ctx->stream>>>(a);
    LDGA_LAUNCHED(ctx, "k_bse_lu32");
    return LDGA_OK;
}

template <int N, int TR, int TC, int WPC, int MINB>
int run_warp32(ldga_ctx* ctx, const BseArgs& a0) {
    BseArgs a = a0;
    const int threads = 32 * WPC;
    const size_t sm = (size_t)N * N * sizeof(double2) + WPC * Warp32Smem<N, TR, TC>::bytes;
    auto kern = k_bse_warp32<N, TR, TC, WPC, MINB>;
    LDGA_CUDA(ctx, set_smem(ctx, kern, sm));
    int chunk = 4 * WPC;
    while (chunk > WPC && (long)((a.nq + chunk - 1) / chunk) * a.nw < 8 * 148) chunk -= WPC;
    a.qchunk = chunk;
    dim3 grid((a.nq + chunk - 1) / chunk, a.nw);
    StageTimer st_(ctx, LDGA_STAGE_BSE);
    kern<<<grid, threads, sm, ctx->stream>>>(a);
    LDGA_LAUNCHED(ctx, "k_bse_warp32");
    return LDGA_OK;
}

#include "bse_jacobi.cuh"

// ------------------------------------------------------------------------------------------------
// Configurations per box size and precision mode (threads per matrix, matrices per CTA, resident
// CTAs per SM the register allocation must allow).  Entry 0 of every list is the default; the
// autotuner (ldga_autotune_bse) times all entries on the handle's own data and records the fastest.
using BseRun = int (*)(ldga_ctx*, const BseArgs&);
using BseRunPair = int (*)(ldga_ctx*, const BseArgs&, const BseArgs&);
template <int N, int LPQ, int MINB, int QPL = 1, bool GSM = true, bool TC = false, bool DM = false, bool P2 = false,
          bool NS = false, int NL = N, bool ADJ = false>
int run_iter_impl(ldga_ctx* ctx, const BseArgs& a, const BseArgs* a_d) {
    if (!ctx->d_qperm) return ctx_fail(ctx, LDGA_ERR_ARG, "preconditioned BSE: q order buffer missing");
    using S = IterSmem<N, GSM, TC, kIterQ * LPQ / QPL / 32, DM, NS>;
    auto kern = k_bse_iter<N, LPQ, QPL, MINB, GSM, TC, DM, P2, NS, NL, ADJ>;
    LDGA_CUDA(ctx, set_smem(ctx, kern, S::bytes));
    StageTimer st_(ctx, LDGA_STAGE_BSE);
    // the q order depends on chi0 only: the second channel of the same bubble reuses it
    if (ctx->qperm_gen != ctx->chi0_gen) {
        if (a.nq <= 4096) {
            int P = 32;
            while (P < a.nq) P <<= 1;
            const size_t smq = (size_t)P * (sizeof(double) + sizeof(int));
            LDGA_CUDA(ctx, set_smem(ctx, k_bse_qorder, smq));
            k_bse_qorder<<<a.nw, 1024, smq, ctx->stream>>>(a.nq, NL, a.chi0, ctx->d_qperm);
            LDGA_LAUNCHED(ctx, "k_bse_qorder");
        } else {
            k_bse_qorder_id<<<148, 256, 0, ctx->stream>>>(a.nq, a.nw, ctx->d_qperm);
            LDGA_LAUNCHED(ctx, "k_bse_qorder_id");
        }
        ctx->qperm_gen = ctx->chi0_gen;
    }
    dim3 grid((a.nq + kIterQ - 1) / kIterQ, a.nw, a_d ? 2 : 1);
    kern<<<grid, kIterQ * LPQ / QPL, S::bytes, ctx->stream>>>(a, a_d ? *a_d : a, ctx->d_qperm);
    LDGA_LAUNCHED(ctx, "k_bse_iter");
    return LDGA_OK;
}

template <int N, int LPQ, int MINB, int QPL = 1, bool GSM = true, bool TC = false, bool DM = false, bool P2 = false,
          bool NS = false, int NL = N>
int run_iter(ldga_ctx* ctx, const BseArgs& a) {
    return run_iter_impl<N, LPQ, MINB, QPL, GSM, TC, DM, P2, NS, NL>(ctx, a, nullptr);
}

template <int N, int LPQ, int MINB, int QPL = 1, bool GSM = true, bool TC = false, bool DM = false, bool P2 = false,
          bool NS = false, int NL = N>
int run_iter_pair(ldga_ctx* ctx, const BseArgs& a_m, const BseArgs& a_d) {
    return run_iter_impl<N, LPQ, MINB, QPL, GSM, TC, DM, P2, NS, NL>(ctx, a_m, &a_d);
}

struct BseVariant {
    BseRun run;
    const char* name;
    BseRunPair run_pair = nullptr;   // both channels in one launch (the preconditioned solve)
};

#define LDGA_SMALL_BOX(N)                                                                              \
    const BseVariant fp64_##N[] = {{&run_lu<N, 8, 1, 2>, "lu8:2"}, {&run_lu<N, 8, 1, 4>, "lu8:4"},     \
                                   {&run_lu<N, 8, 1, 8>, "lu8:8"}};                                     \
    const BseVariant mixed_##N[] = {{&run_warp32<N, 8, 4, 4, 1>, "warp:1"},                            \
                                    {&run_warp32<N, 8, 4, 4, 3>, "warp:3"}};                           \
    const BseVariant inv_##N[] = {{&run_tile<N, 8, 8, 2, 1, double, LDGA_PREC_FP64_INV>, "gj8x2"}};
LDGA_SMALL_BOX(4)
LDGA_SMALL_BOX(6)
LDGA_SMALL_BOX(8)
LDGA_SMALL_BOX(10)
LDGA_SMALL_BOX(12)
#undef LDGA_SMALL_BOX
// Nν = 16..30: the warp LU stays the MIXED default (its N^3 is small); the q-shared preconditioned
// iteration is a configuration the autotuner may pick
// ...and the tensor-core preconditioned iteration (both products on tensor cores, the group inverse
// on tcgen05) on tiles of NP >= N rows, NP a multiple of 8, as a candidate: with few q per ω its
// groups are wide, so the autotuner decides
#define LDGA_ITER_BOX(N, LPQ, MINB, NP, MINB_TC, TCNAME)                                                \
    const BseVariant fp64_##N[] = {{&run_lu<N, 8, 1, 2>, "lu8:2"}, {&run_lu<N, 8, 1, 4>, "lu8:4"},     \
                                   {&run_lu<N, 8, 1, 8>, "lu8:8"}};                                     \
    const BseVariant mixed_##N[] = {{&run_warp32<N, 8, 4, 4, 1>, "warp:1"}, {&run_warp32<N, 8, 4, 4, 3>, "warp:3"}, \
                                    {&run_iter<N, LPQ, MINB>, "iter"},                                 \
                                    {&run_iter<NP, 8, MINB_TC, 2, true, true, true, true, true, N>, TCNAME, \
                                     &run_iter_pair<NP, 8, MINB_TC, 2, true, true, true, true, true, N>}}; \
    const BseVariant inv_##N[] = {{&run_tile<N, 8, 8, 2, 1, double, LDGA_PREC_FP64_INV>, "gj8x2"}};
LDGA_ITER_BOX(16, 4, 4, 16, 4, "iter8x2dm2ns16:4")
LDGA_ITER_BOX(20, 4, 4, 24, 4, "iter8x2dm2ns24:4")
LDGA_ITER_BOX(30, 4, 3, 32, 3, "iter8x2dm2ns32:3")
#undef LDGA_ITER_BOX
const BseVariant fp64_40[] = {{&run_lu<40, 8, 1, 6>, "lu8:6"}, {&run_lu<40, 8, 1, 4>, "lu8:4"},
                              {&run_lu<40, 8, 1, 5>, "lu8:5"}};
// the default: the group inverse by Newton-Schulz on tcgen05 tensor cores (Gauss-Jordan as its fallback)
const BseVariant mixed_40[] = {{&run_iter<40, 8, 3, 2, true, true, true, true, true>, "iter8x2dm2ns:3",
                                &run_iter_pair<40, 8, 3, 2, true, true, true, true, true>},
                               {&run_iter<40, 8, 3, 2, true, true, true, true>, "iter8x2dm2:3", &run_iter_pair<40, 8, 3, 2, true, true, true, true>},
                               {&run_iter<40, 8, 2, 2, true, true, true, true>, "iter8x2dm2:2", &run_iter_pair<40, 8, 2, 2, true, true, true, true>},
                               {&run_iter<40, 8, 3, 2, true, true, true>, "iter8x2dm:3", &run_iter_pair<40, 8, 3, 2, true, true, true>},
                               {&run_iter<40, 8, 2, 2, true, true, true>, "iter8x2dm:2", &run_iter_pair<40, 8, 2, 2, true, true, true>},
                               {&run_iter<40, 8, 3, 2, true, true>, "iter8x2tc:3"}, {&run_iter<40, 8, 2, 2, true, true>, "iter8x2tc:2"},
                               {&run_iter<40, 8, 2, 2>, "iter8x2:2"}, {&run_iter<40, 8, 3, 2>, "iter8x2:3"},
                               {&run_iter<40, 8, 2>, "iter8:2"}, {&run_iter<40, 4, 3>, "iter"},
                               {&run_warp32<40, 8, 4, 4, 3>, "warp:3"}, {&run_warp32<40, 8, 4, 4, 2>, "warp:2"}};
const BseVariant inv_40[] = {{&run_tile<40, 8, 8, 2, 1, double, LDGA_PREC_FP64_INV>, "gj8x2"}};
const BseVariant fp64_60[] = {{&run_lu<60, 16, 1, 2>, "lu16:2"}, {&run_lu<60, 16, 1, 1>, "lu16:1"},
                              {&run_lu<60, 16, 1, 3>, "lu16:3"}};
// MIXED may pick any configuration whose results meet the FP64 backward-error bound, the FP64 LU
// included: at Nν = 60 and 120 that is the fastest one measured
// the preconditioned iteration on tiles padded to 64 (an identity block below the box), both products
// on tensor cores and the group inverse on tcgen05, one 128-thread CTA per SM (151 KB of shared memory)
const BseVariant mixed_60[] = {{&run_iter<64, 8, 1, 2, true, true, true, true, true, 60>, "iter8x2dm2ns64:1",
                                &run_iter_pair<64, 8, 1, 2, true, true, true, true, true, 60>},
                               {&run_lu<60, 16, 1, 2>, "lu16:2"}, {&run_lu32<60, 16, 1, 3>, "lu32x16:3"},
                               {&run_lu32<60, 16, 1, 2>, "lu32x16:2"}, {&run_iter<60, 8, 1>, "iter"}};
const BseVariant inv_60[] = {{&run_tile<60, 16, 16, 1, 1, double, LDGA_PREC_FP64_INV>, "gj16x1"}};
// Nν = 120: Gamma(w) (230 KB) exceeds shared memory and is read through L1/L2; FP64_INV solves by LU
// (32 x 32 threads per matrix -- a 4 x 4 register tile instead of 16 x 16 threads' spilling 8 x 8 --
// measured 1.76x slower: 120 steps of a 1024-thread barrier over little work per thread)
const BseVariant fp64_120[] = {{&run_lu<120, 16, 1, 1, false>, "lu16g:1"}};
// MIXED at Nν = 120: the Jacobi refinement (bse_jacobi.cuh), whose stop test bounds the forward error
// too (the test matrices' condition numbers reach 1e4, where a backward error of 1e-14 alone would
// not guarantee the 1e-10 forward accuracy), then the LU forms
const BseVariant mixed_120[] = {{&run_jacobi<120, 32, 4, true>, "jac", &run_jacobi_pair<120, 32, 4, true>},
                                {&run_jacobi<120, 32, 4, false>, "jac4", &run_jacobi_pair<120, 32, 4, false>},
                                {&run_jacobi<120, 16, 2, true>, "jac16:2", &run_jacobi_pair<120, 16, 2, true>},
                                {&run_lu<120, 16, 1, 1, false>, "lu16g:1"}, {&run_lu32<120, 16, 1, 1, false>, "lu32x16g:1"}};

int variants_of(int nnu, int prec, const BseVariant** out) {
#define LDGA_BOX(N)                                                                                      \
    case N:                                                                                             \
        if (prec == LDGA_PREC_FP64) { *out = fp64_##N; return (int)(sizeof(fp64_##N) / sizeof(BseVariant)); }     \
        if (prec == LDGA_PREC_MIXED) { *out = mixed_##N; return (int)(sizeof(mixed_##N) / sizeof(BseVariant)); }  \
        *out = inv_##N; return (int)(sizeof(inv_##N) / sizeof(BseVariant));
    switch (nnu) {
        LDGA_BOX(4) LDGA_BOX(6) LDGA_BOX(8) LDGA_BOX(10) LDGA_BOX(12) LDGA_BOX(16) LDGA_BOX(20) LDGA_BOX(30)
        LDGA_BOX(40) LDGA_BOX(60)
        case 120:
            if (prec == LDGA_PREC_MIXED) { *out = mixed_120; return (int)(sizeof(mixed_120) / sizeof(BseVariant)); }
            *out = fp64_120; return (int)(sizeof(fp64_120) / sizeof(BseVariant));
        default: *out = nullptr; return 0;
    }
#undef LDGA_BOX
}

// chosen variant per (Nν, precision mode); absent = 0
std::mutex g_tune_mu;
std::map<std::pair<int, int>, int> g_tune;

int tuned_index(int nnu, int prec) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find({nnu, prec});
    return it == g_tune.end() ? 0 : it->second;
}

// The kernels see the ω shard as a whole problem of shard_nw frequencies: every array has ω as its
// slowest index, so the shard is the same arrays advanced to w_lo.
BseArgs bse_args(ldga_ctx* ctx, int channel) {
    BseArgs a;
    const size_t w0 = (size_t)ctx->w_lo, nq = (size_t)ctx->Nq, nnu = (size_t)ctx->Nnu;
    a.nq = ctx->Nq; a.nnu = ctx->Nnu; a.nw = shard_nw(ctx); a.qchunk = 1;
    a.beta = ctx->mp.beta; a.U = ctx->mp.U;
    a.s = channel == LDGA_CH_D ? -1 : 1;
    a.Gamma = ctx->d_Gamma[channel] + w0 * nnu * nnu;
    a.chi0 = ctx->d_chi0 + w0 * nq * nnu;
    a.chi = ctx->d_chi[channel] + w0 * nq;
    a.gam = ctx->d_gam[channel] + w0 * nq * nnu;
    a.flags = ctx->d_flags + w0 * nq;
    a.stats = ctx->d_iter_stats;
    a.max_sweeps = ctx->iter_sweeps;
    return a;
}

// ---- MIXED adjoint at Nν = 40: the transposed systems (Gamma(w) + diag(1/chi0)) conj(z) = conj(y_bar)
// by the preconditioned iteration (k_bse_iter<..., ADJ>) on a transposed copy of Gamma, with the
// pivot-free FP64 LU adjoint (k_bse_adj, list mode) for the matrices it leaves above its bound.
// The same formulas as k_bse_adj, split around the solve:
//   k_adj_rhs:     y = gamma chi0 / rf -> ybuf; conj(y_bar) -> zbuf (the right-hand side)
//   k_bse_iter:    zbuf <- z = conj(x) for the solved matrices, flags 1 for the others
//   k_adj_chi0bar: chi0_bar from y, z for the unflagged matrices (k_bse_adj writes the others)

// dst[w][i N + j] = src[w][j N + i]
__global__ void k_transpose_gamma(int n, int nw, const double2* __restrict__ src, double2* __restrict__ dst) {
    const size_t tot = (size_t)n * n * nw;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < tot; e += (size_t)gridDim.x * blockDim.x) {
        const size_t w = e / ((size_t)n * n);
        const int r = (int)(e - w * n * n), i = r / n, j = r - (r / n) * n;
        dst[e] = src[w * n * n + (size_t)j * n + i];
    }
}

// one thread per (q, w): two sweeps over nu (q fastest in memory, so the warp's loads coalesce)
__global__ void k_adj_rhs(const BseAdjArgs a) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;   // q + Nq w
    if (e >= a.nq * a.nw) return;
    const int q = e % a.nq, w = e / a.nq, n = a.nnu;
    const double f = 1.0 + a.s * a.U * a.chi[e], rf = 1.0 / f;
    double s1 = 0.0;
    for (int i = 0; i < n; ++i) {
        const size_t ci = (size_t)q + (size_t)a.nq * (i + (size_t)n * w);
        const double2 c0 = a.chi0[ci];
        const double2 y = cscale(cmul(a.gam[ci], c0), f);
        a.ybuf[ci] = y;
        if (a.gam_bar) {
            const double2 gb = a.gam_bar[ci], yd = cmul(y, cinv(c0));
            s1 += gb.x * yd.x + gb.y * yd.y;             // Re(conj(gb) y d)
        }
    }
    const double xbar = (a.chi_bar ? a.chi_bar[e] : 0.0) - a.s * a.U * rf * rf * s1;
    for (int i = 0; i < n; ++i) {
        const size_t ci = (size_t)q + (size_t)a.nq * (i + (size_t)n * w);
        double2 yb = make_double2(xbar / (a.beta * a.beta), 0.0);
        if (a.gam_bar) yb = cadd(yb, cmul(cconj(cscale(cinv(a.chi0[ci]), rf)), a.gam_bar[ci]));
        a.zbuf[ci] = cconj(yb);
    }
}

// one thread per (q, nu, w) of an unflagged matrix
__global__ void k_adj_chi0bar(const BseAdjArgs a) {
    const size_t tot = (size_t)a.nq * a.nnu * a.nw;
    for (size_t ci = blockIdx.x * (size_t)blockDim.x + threadIdx.x; ci < tot; ci += (size_t)gridDim.x * blockDim.x) {
        const int q = (int)(ci % a.nq);
        const size_t w = ci / ((size_t)a.nq * a.nnu);
        const size_t cq = (size_t)q + (size_t)a.nq * w;
        if (a.flags[cq] != 0) continue;
        const double rf = 1.0 / (1.0 + a.s * a.U * a.chi[cq]);
        const double2 z = a.zbuf[ci], y = a.ybuf[ci], d = cinv(a.chi0[ci]);
        double2 db = cscale(cmul(z, cconj(y)), -1.0);
        if (a.gam_bar) db = cadd(db, cmul(cconj(cscale(y, rf)), a.gam_bar[ci]));
        const double2 c0b = cscale(cmul(cconj(cmul(d, d)), db), -1.0);
        a.chi0_bar[ci] = a.accumulate ? cadd(a.chi0_bar[ci], c0b) : c0b;
    }
}

}  // namespace

bool bse_has_fast_path(int nnu) {
    switch (nnu) {
        case 4: case 6: case 8: case 10: case 12: case 16: case 20: case 30: case 40: case 60: case 120: return true;
        default: return false;
    }
}

size_t bse_pivot_smem(int nnu) { return (size_t)nnu * (nnu + 1) * sizeof(double2) + 64 * sizeof(double) + 16; }

int bse_variant_count(int nnu, int prec) {
    const BseVariant* v = nullptr;
    return variants_of(nnu, prec, &v);
}

const char* bse_variant_name(int nnu, int prec, int i) {
    const BseVariant* v = nullptr;
    const int n = variants_of(nnu, prec, &v);
    return (i >= 0 && i < n) ? v[i].name : nullptr;
}

int bse_tuned_variant(int nnu, int prec) { return tuned_index(nnu, prec); }

void bse_set_variant(int nnu, int prec, int i) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[{nnu, prec}] = i;
}

void bse_reset_variants() {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune.clear();
}

int bse_run_variant(ldga_ctx* ctx, int channel, int i) {
    const BseVariant* v = nullptr;
    const int n = variants_of(ctx->Nnu, ctx->prec, &v);
    if (i < 0 || i >= n) return ctx_fail(ctx, LDGA_ERR_ARG, "BSE variant index out of range");
    return v[i].run(ctx, bse_args(ctx, channel));
}

int launch_bse(ldga_ctx* ctx, int channel, int32_t* d_fail) {
    const BseArgs a = bse_args(ctx, channel);
    const int n = ctx->Nq * shard_nw(ctx);
    int st = LDGA_OK;
    bool generic = false;
    {
        const BseVariant* v = nullptr;
        const int nv = variants_of(ctx->Nnu, ctx->prec, &v);
        if (nv > 0) {
            int i = tuned_index(ctx->Nnu, ctx->prec);
            if (i >= nv) i = 0;
            st = v[i].run(ctx, a);
        } else {
            generic = true;
        }
    }
    if (st != LDGA_OK) return st;
    const bool in_hbm = bse_pivot_smem(ctx->Nnu) > LDGA_PIVOT_SMEM_MAX;
    if (in_hbm && !ctx->d_pivot_scratch) return ctx_fail(ctx, LDGA_ERR_ARG, "pivoted BSE scratch missing");
    const size_t smp = in_hbm ? 64 * sizeof(double) + 16 : bse_pivot_smem(ctx->Nnu);
    double2* gscr = in_hbm ? ctx->d_pivot_scratch : nullptr;
    LDGA_CUDA(ctx, set_smem(ctx, k_bse_lu_pivot, smp));
    if (generic) {
        StageTimer st_(ctx, LDGA_STAGE_BSE_FALLBACK);
        k_bse_lu_pivot<<<LDGA_PIVOT_GRID, 256, smp, ctx->stream>>>(a, nullptr, n, nullptr, gscr);
        LDGA_LAUNCHED(ctx, "k_bse_lu_pivot");
    } else {
        // flagged matrices: compacted on the device, re-solved by a grid-stride pivoted kernel that reads
        // the count from device memory (zero work when nothing was flagged)
        LDGA_CUDA(ctx, cudaMemsetAsync(ctx->d_count, 0, sizeof(int32_t), ctx->stream));
        k_compact_flags<<<148, 256, 0, ctx->stream>>>(a.flags, n, ctx->d_list, ctx->d_count);
        LDGA_LAUNCHED(ctx, "k_compact_flags");
        StageTimer st_(ctx, LDGA_STAGE_BSE_FALLBACK);
        k_bse_lu_pivot<<<LDGA_PIVOT_GRID, 256, smp, ctx->stream>>>(a, ctx->d_list, 0, ctx->d_count, gscr);
        LDGA_LAUNCHED(ctx, "k_bse_lu_pivot");
    }
    // matrices that stayed non-finite after the pivoted solve, accumulated into *d_fail
    k_count_flags<<<148, 256, 0, ctx->stream>>>(a.flags, n, d_fail);
    LDGA_LAUNCHED(ctx, "k_count_flags");
    return LDGA_OK;
}

// Both channels of the chain: one launch of the tuned configuration when it has a two-channel form
// (channel d flags into d_flags2); the matrices it leaves above its backward-error bound are appended
// to one list per channel (counts in d_count[2], d_count[3], zeroed by the caller with d_fail) and
// re-solved by one pivoted launch over both lists.  Otherwise launch_bse for m, then d.
int launch_bse_pair(ldga_ctx* ctx, int32_t* d_fail) {
    const BseVariant* v = nullptr;
    const int nv = variants_of(ctx->Nnu, ctx->prec, &v);
    int i = nv > 0 ? tuned_index(ctx->Nnu, ctx->prec) : 0;
    if (i >= nv) i = 0;
    if (nv == 0 || !v[i].run_pair) {
        const int st = launch_bse(ctx, LDGA_CH_M, d_fail);
        return st != LDGA_OK ? st : launch_bse(ctx, LDGA_CH_D, d_fail);
    }
    const size_t nall = (size_t)ctx->Nq * ctx->Nw;
    if (!ctx->d_flags2) {
        LDGA_CUDA(ctx, cudaMalloc(reinterpret_cast<void**>(&ctx->d_flags2), nall * sizeof(int32_t)));
        LDGA_CUDA(ctx, cudaMemsetAsync(ctx->d_flags2, 0, nall * sizeof(int32_t), ctx->stream));
    }
    if (!ctx->d_list2) LDGA_CUDA(ctx, cudaMalloc(reinterpret_cast<void**>(&ctx->d_list2), nall * sizeof(int32_t)));
    BseArgs am = bse_args(ctx, LDGA_CH_M), ad = bse_args(ctx, LDGA_CH_D);
    ad.flags = ctx->d_flags2 + (size_t)ctx->w_lo * ctx->Nq;
    am.fail_list = ctx->d_list;
    am.fail_count = ctx->d_count + 2;
    ad.fail_list = ctx->d_list2;
    ad.fail_count = ctx->d_count + 3;
    const int st = v[i].run_pair(ctx, am, ad);
    if (st != LDGA_OK) return st;
    const bool in_hbm = bse_pivot_smem(ctx->Nnu) > LDGA_PIVOT_SMEM_MAX;
    if (in_hbm && !ctx->d_pivot_scratch) return ctx_fail(ctx, LDGA_ERR_ARG, "pivoted BSE scratch missing");
    const size_t smp = in_hbm ? 64 * sizeof(double) + 16 : bse_pivot_smem(ctx->Nnu);
    double2* gscr = in_hbm ? ctx->d_pivot_scratch : nullptr;
    LDGA_CUDA(ctx, set_smem(ctx, k_bse_lu_pivot_pair, smp));
    StageTimer st_(ctx, LDGA_STAGE_BSE_FALLBACK);
    k_bse_lu_pivot_pair<<<LDGA_PIVOT_GRID, 256, smp, ctx->stream>>>(am, ad, gscr, d_fail);
    LDGA_LAUNCHED(ctx, "k_bse_lu_pivot_pair");
    return LDGA_OK;
}

int launch_bse_adj(ldga_ctx* ctx, int channel, const double* chi_bar, const double2* gam_bar, double2* chi0_bar,
                   double2* ybuf, double2* zbuf, double2* gamma_bar, int32_t* d_fail, bool accumulate) {
    BseAdjArgs a;
    a.nq = ctx->Nq; a.nnu = ctx->Nnu; a.nw = ctx->Nw; a.qchunk = 1;
    a.beta = ctx->mp.beta; a.U = ctx->mp.U;
    a.s = channel == LDGA_CH_D ? -1 : 1;
    a.Gamma = ctx->d_Gamma[channel];
    a.chi0 = ctx->d_chi0;
    a.chi = ctx->d_chi[channel];
    a.gam = ctx->d_gam[channel];
    a.chi_bar = chi_bar; a.gam_bar = gam_bar;
    a.chi0_bar = chi0_bar; a.ybuf = ybuf; a.zbuf = zbuf;
    a.accumulate = accumulate ? 1 : 0;
    a.flags = ctx->d_flags;
    int st = LDGA_OK;
    if (ctx->prec == LDGA_PREC_MIXED && ctx->Nnu == 40) {
        // MIXED: the preconditioned iteration on the transposed systems, the LU for what it leaves
        constexpr int N = 40;
        const size_t vvw = (size_t)N * N * ctx->Nw;
        if (!ctx->d_gamma_t) {
            if (ctx->capturing) return ctx_fail(ctx, LDGA_ERR_STATE, "BSE adjoint: scratch not allocated before capture");
            LDGA_CUDA(ctx, cudaMalloc(reinterpret_cast<void**>(&ctx->d_gamma_t), vvw * sizeof(double2)));
        }
        k_transpose_gamma<<<2 * 148, 256, 0, ctx->stream>>>(N, ctx->Nw, ctx->d_Gamma[channel], ctx->d_gamma_t);
        LDGA_LAUNCHED(ctx, "k_transpose_gamma");
        const int nqw = ctx->Nq * ctx->Nw;
        k_adj_rhs<<<(nqw + 255) / 256, 256, 0, ctx->stream>>>(a);
        LDGA_LAUNCHED(ctx, "k_adj_rhs");
        BseArgs b = bse_args(ctx, channel);
        b.Gamma = ctx->d_gamma_t;
        b.rhs = zbuf;
        b.gam = zbuf;
        b.chi = nullptr;
        b.stats = nullptr;
        b.fail_list = ctx->d_list;
        b.fail_count = ctx->d_count + 2;
        LDGA_CUDA(ctx, cudaMemsetAsync(ctx->d_count + 2, 0, sizeof(int32_t), ctx->stream));
        st = run_iter_impl<N, 8, 2, 2, true, true, true, true, true, N, true>(ctx, b, nullptr);
        if (st != LDGA_OK) return st;
        // chi0_bar of the solved matrices first: the LU below clears the flags of those it solves
        k_adj_chi0bar<<<4 * 148, 256, 0, ctx->stream>>>(a);
        LDGA_LAUNCHED(ctx, "k_adj_chi0bar");
        BseAdjArgs al = a;
        al.list = ctx->d_list;
        al.count = ctx->d_count + 2;
        const size_t sm = (size_t)N * N * sizeof(double2) + LuSmem<N, 8>::bytes + 2 * N * sizeof(double2) + 16;
        auto kern = k_bse_adj<N, 8, 6>;
        LDGA_CUDA(ctx, set_smem(ctx, kern, sm));
        kern<<<LDGA_PIVOT_GRID, 64, sm, ctx->stream>>>(al);
        LDGA_LAUNCHED(ctx, "k_bse_adj");
    } else {
    switch (ctx->Nnu) {
        case 4: st = run_bse_adj<4, 8, 4>(ctx, a); break;
        case 6: st = run_bse_adj<6, 8, 4>(ctx, a); break;
        case 8: st = run_bse_adj<8, 8, 4>(ctx, a); break;
        case 10: st = run_bse_adj<10, 8, 4>(ctx, a); break;
        case 12: st = run_bse_adj<12, 8, 4>(ctx, a); break;
        case 16: st = run_bse_adj<16, 8, 4>(ctx, a); break;
        case 20: st = run_bse_adj<20, 8, 4>(ctx, a); break;
        case 30: st = run_bse_adj<30, 8, 4>(ctx, a); break;
        case 40: st = run_bse_adj<40, 8, 6>(ctx, a); break;
        case 60: st = run_bse_adj<60, 16, 2>(ctx, a); break;
        default: return ctx_fail(ctx, LDGA_ERR_ARG, "BSE adjoint: fermionic box " + std::to_string(ctx->Nnu) +
                                                        " not built (4..60 even sizes of the tiled kernels)");
    }
    }
    if (st != LDGA_OK) return st;
    const int n = ctx->Nnu;
    dim3 g2((n + 31) / 32, (n + 31) / 32, ctx->Nw);
    k_bse_gamma_grad<<<g2, 256, 0, ctx->stream>>>(ctx->Nq, n, ybuf, zbuf, gamma_bar);
    LDGA_LAUNCHED(ctx, "k_bse_gamma_grad");
    k_count_flags<<<148, 256, 0, ctx->stream>>>(ctx->d_flags, ctx->Nq * ctx->Nw, d_fail);
    LDGA_LAUNCHED(ctx, "k_count_flags");
    return LDGA_OK;
}

// ------------------------------------------------------------------------------------------------
// Self-test of the tcgen05 Newton-Schulz group inverse (ns_inverse.cuh), one CTA of 128 threads on
// an N x N complex matrix b (row-major float2) and seed x0.  its >= 0: its iterations from x0, x_out
// = the iterate, err_out[0] = max_i sum_j |I - b X|_ij of the iterate before the last update (0 when
// its = 0); its < 0: x_out = the single product b x0 (both factors rounded to TF32).
namespace {

template <int N>
struct NsTestSmem {
    using S = ns::NsSmem<N>;
    // 4 KB beyond the operand buffers: every byte the descriptors can address stays inside the
    // allocation whichever of the two strides the hardware applies to rows
    static constexpr uint32_t off_bar = S::bytes + 4096, off_slot = off_bar + 8, off_red = off_bar + 16;
    static constexpr uint32_t bytes = off_red + 64;
};

template <int N>
__global__ void __launch_bounds__(128) k_ns_selftest(const float2* __restrict__ b, const float2* __restrict__ x0,
                                                      int its, float2* __restrict__ xout, float* __restrict__ err,
                                                      int32_t* __restrict__ status) {
    using S = ns::NsSmem<N>;
    using T = NsTestSmem<N>;
    extern __shared__ __align__(128) unsigned char ns_raw[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(ns_raw + T::off_bar);
    uint32_t* slot = reinterpret_cast<uint32_t*>(ns_raw + T::off_slot);
    float* red = reinterpret_cast<float*>(ns_raw + T::off_red);
    const int tid = threadIdx.x, warp = tid >> 5;
    if (tid == 0) {
        tc05::mbar_init(bar, 1);
        tc05::mbar_fence_init();
    }
    if (warp == 0) tc05::tmem_alloc(slot, S::tmem_cols);
    if (tid < N) {
        for (int k = 0; k < N; k += 4) {
            float v[4][4];
            for (int u = 0; u < 4; ++u) {
                const float2 bb = b[tid * N + k + u], xx = x0[tid * N + k + u];
                v[0][u] = bb.x; v[1][u] = bb.y; v[2][u] = xx.x; v[3][u] = xx.y;
            }
            ns::store_a4<N>(ns_raw + S::off_br, tid, k, v[0][0], v[0][1], v[0][2], v[0][3]);
            ns::store_a4<N>(ns_raw + S::off_bi, tid, k, v[1][0], v[1][1], v[1][2], v[1][3]);
            ns::store_a4<N>(ns_raw + S::off_xr, tid, k, v[2][0], v[2][1], v[2][2], v[2][3]);
            ns::store_a4<N>(ns_raw + S::off_xi, tid, k, v[3][0], v[3][1], v[3][2], v[3][3]);
            for (int u = 0; u < 4; ++u) {
                ns::store_b<N>(ns_raw + S::off_tr, tid, k + u, v[2][u]);
                ns::store_b<N>(ns_raw + S::off_ti, tid, k + u, v[3][u]);
            }
        }
        if (its == 0)
            for (int j = 0; j < N; ++j) xout[tid * N + j] = x0[tid * N + j];
    }
    tc05::fence_before();
    __syncthreads();
    tc05::fence_after();
    ns::NsState st{*slot, 0u, true};
    float e = 0.f;
    auto emit = [&](int t, int c, const float (&re)[16], const float (&im)[16]) {
        for (int j = 0; j < 16; ++j)
            if (c + j < N) xout[t * N + c + j] = make_float2(re[j], im[j]);
    };
    if (its > 0) {
        ns::newton_schulz<N>(ns_raw, bar, red, st, its, 0.f, emit, &e);
    } else if (its < 0) {
        const uint32_t base = tc05::smem_addr(ns_raw);
        ns::product<N>(st, bar, base + S::off_br, base + S::off_bi, base + S::off_tr, base + S::off_ti);
        if (warp < (N + 31) / 32) {
            for (int c = 0; c < N; c += 16) {
                float re[16], im[16];
                ns::load_chunk(st.tmem + ((uint32_t)(32 * warp) << 16), c, re, im);
                if (tid < N) emit(tid, c, re, im);
            }
        }
    }
    ns::drain(st, bar);
    tc05::fence_before();
    __syncthreads();
    if (warp == 0) {
        tc05::fence_after();
        tc05::tmem_free(st.tmem, S::tmem_cols);
    }
    if (tid == 0) {
        err[0] = e;
        status[0] = st.ok ? 0 : 1;
    }
}

}  // namespace

extern "C" int ldga_selftest_group_inverse(int32_t n, const float* b, const float* x0, int32_t its, float* x_out,
                                           float* err_out) {
    if (n != 40 || !b || !x0 || !x_out || !err_out || its > 16) return LDGA_ERR_ARG;
    using T = NsTestSmem<40>;
    const size_t mb = (size_t)n * n * 2 * sizeof(float);
    float2 *db = nullptr, *dx = nullptr, *dout = nullptr;
    float* derr = nullptr;
    int32_t* dst = nullptr;
    int rc = LDGA_OK;
    int32_t status = 0;
    float err = 0.f;
    if (cudaMalloc(&db, mb) != cudaSuccess || cudaMalloc(&dx, mb) != cudaSuccess || cudaMalloc(&dout, mb) != cudaSuccess ||
        cudaMalloc(&derr, sizeof(float)) != cudaSuccess || cudaMalloc(&dst, sizeof(int32_t)) != cudaSuccess) {
        rc = LDGA_ERR_CUDA;
    }
    if (rc == LDGA_OK && (cudaMemcpy(db, b, mb, cudaMemcpyHostToDevice) != cudaSuccess ||
                          cudaMemcpy(dx, x0, mb, cudaMemcpyHostToDevice) != cudaSuccess))
        rc = LDGA_ERR_CUDA;
    if (rc == LDGA_OK) {
        auto kern = k_ns_selftest<40>;
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T::bytes) != cudaSuccess) {
            rc = LDGA_ERR_CUDA;
        } else {
            kern<<<1, 128, T::bytes>>>(db, dx, its, dout, derr, dst);
            if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) rc = LDGA_ERR_CUDA;
        }
    }
    if (rc == LDGA_OK && (cudaMemcpy(x_out, dout, mb, cudaMemcpyDeviceToHost) != cudaSuccess ||
                          cudaMemcpy(&err, derr, sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess ||
                          cudaMemcpy(&status, dst, sizeof(int32_t), cudaMemcpyDeviceToHost) != cudaSuccess))
        rc = LDGA_ERR_CUDA;
    cudaFree(db); cudaFree(dx); cudaFree(dout); cudaFree(derr); cudaFree(dst);
    if (rc != LDGA_OK) return rc;
    err_out[0] = err;
    return status == 0 ? LDGA_OK : LDGA_ERR_NUMERIC;
}
