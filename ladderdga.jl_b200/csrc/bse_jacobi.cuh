// MIXED BSE for the large box (Nν = 120, the β = 40 points of an uneven batch): Jacobi-preconditioned
// iterative refinement, FP64 throughout.  Included by kernels_bse.cu inside its anonymous namespace:
// it uses BseArgs, the complex helpers and mma_f64 defined there.
//
// calc_χγ solves B_q x = 1 with B_q = Γ(ω)ᵀ + diag(1/χ₀(q, :, ω)) for every (q, ω) (BSETools.jl:219-238).
// At Nν = 120 the diagonal dominates each row of B_q (the row sums of |B_ij / B_jj| off the diagonal
// stay below 0.05 on these points).  So the iteration
//     r = 1 - B_q x,   x += diag(B_q)^-1 r,   from x = diag(B_q)^-1 1,
// contracts by that factor per sweep.  A q stops when two bounds hold: the FP64 backward error of
// the other MIXED kernels (at most 1e-14), and a forward-error bound that does not depend on the
// condition number of B_q.  With theta_q = max_i sum_{j != i} |B_ij| / |B_ii| < 1 (bounded from the
// row sums), |x* - x| <= |dx| / (1 - theta_q) for the next correction dx.  That bound must be at
// most 1e-14 |x|.  On the β = 40 points this takes 5.5 sweeps on average, at most 6.  A q still
// above either bound after max_sweeps sweeps is flagged for the pivoted FP64 solve; a pair launch
// also appends it to its channel's list.
//
// Γ(ω) is 230 KB and does not fit shared memory.  A CTA therefore takes 32 q of one ω and streams
// Γ(ω) from L2 once per sweep, in tiles of 8 columns (cp.async, double-buffered).  All 32 q use
// every tile:
//     R = Γᵀ X  (N × 32 complex),
// as FP64 tensor-core products (mma.sync m8n8k4 .f64).  The default (K3, Karatsuba) takes three
// real products per complex tile: S1 = Re·Re, S2 = Im·Im, S3 = (Re + Im)·(Re + Im), then
// Re = S1 - S2 and Im = S3 - S1 - S2.  The form with four ("jac4": Re = Σ Re·Re + Im·(-Im),
// Im = Σ Re·Im + Im·Re) needs no FP64 add before a product and one accumulator less.  It does a
// third more tensor work, and measured 10 % slower on the β = 40 points; the autotuner times both.
// A CTA of Q q (32 or 16) runs 3 Q/8 warps: warp (g, n) owns rows [g N/3, (g+1) N/3) (N/24
// m-tiles of 8) of the 8 q of n-tile n.  Lane l of a warp owns rows 8 mt + l/4 and the q pair
// 8 n + 2 (l%4) + {0, 1} of every m-tile mt.  It forms r there and updates x in shared memory;
// reductions over rows run by shuffles within the warp, then over the three row groups through
// shared memory.  Q = 32 runs one CTA per SM with NBUF = 4 tile buffers; Q = 16 runs two CTAs per
// SM, so that one CTA's barriers and epilogue overlap the other's products; Γ then crosses L2
// twice as often per q.
//
// Shared memory (JacSmem): NBUF Γ tiles [N][8] complex; x and D = 1/χ₀, each [N][Q + 2] complex;
// the diagonal of Γ and its off-diagonal row sums [N]; reduction slots.  The fragment loads are
// conflict-free (a 16-byte load serves 8 lanes per wavefront):
//   - a tile row stores its 8 columns XOR-swizzled by 4 on odd rows;
//   - the x and D rows have a stride ≡ 2 (mod 8) complex.
constexpr int kJacKC = 8;             // Γ columns per streamed tile
constexpr double kSqrt2 = 1.4142135623730951;

template <int N, int Q, int NBUF>
struct JacSmem {
    static_assert(N % 24 == 0, "three row groups of whole 8-row tiles");
    static_assert(Q == 16 || Q == 32, "q per CTA");
    static_assert(NBUF >= 2, "double buffering at least");
    static constexpr int MTW = N / 24;                  // m-tiles per warp
    static constexpr int NWN = Q / 8;                   // n-tiles
    static constexpr int WARPS = 3 * NWN;
    static constexpr int THREADS = 32 * WARPS;
    static constexpr int LDX = Q + 2;                   // ≡ 2 (mod 8)
    static constexpr size_t tile = (size_t)N * kJacKC;  // complex per tile
    static constexpr size_t off_g = 0;                                                 // [NBUF][N][8] double2
    static constexpr size_t off_x = off_g + NBUF * tile * sizeof(double2);             // [N][LDX] double2
    static constexpr size_t off_d = off_x + (size_t)N * LDX * sizeof(double2);         // [N][LDX] double2
    static constexpr size_t off_diag = off_d + (size_t)N * LDX * sizeof(double2);      // [N] double2
    static constexpr size_t off_row = off_diag + (size_t)N * sizeof(double2);          // [N] double
    static constexpr size_t off_red = off_row + (size_t)N * sizeof(double);            // [5][3][Q] double
    static constexpr size_t off_conv = off_red + 15 * (size_t)Q * sizeof(double);      // [Q] int
    static constexpr size_t bytes = off_conv + Q * sizeof(int);
};

// element (row i, column c < 8) of a tile
__device__ __forceinline__ int jac_tile_idx(int i, int c) { return i * kJacKC + (c ^ ((i & 1) << 2)); }

__device__ __forceinline__ void jac_cp16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void jac_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int K>
__device__ __forceinline__ void jac_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(K) : "memory"); }

template <int N, int Q, int NBUF, bool K3>
__global__ void __launch_bounds__(JacSmem<N, Q, NBUF>::THREADS, Q == 16 ? 2 : 1)
k_bse_jacobi(const BseArgs a_m, const BseArgs a_d) {
    using S = JacSmem<N, Q, NBUF>;
    constexpr int kJacQ = Q;
    constexpr int kJacThreads = S::THREADS;
    constexpr int kJacWarps = S::WARPS;
    constexpr int NT = N / kJacKC;                     // Γ tiles per sweep
    BseArgs a = a_m;
    if (blockIdx.z) {
        a.s = a_d.s; a.Gamma = a_d.Gamma; a.chi = a_d.chi; a.gam = a_d.gam; a.flags = a_d.flags;
        a.fail_list = a_d.fail_list; a.fail_count = a_d.fail_count;
    }
    extern __shared__ __align__(16) unsigned char jac_raw[];
    double2* G = reinterpret_cast<double2*>(jac_raw + S::off_g);
    double2* X = reinterpret_cast<double2*>(jac_raw + S::off_x);
    double2* D = reinterpret_cast<double2*>(jac_raw + S::off_d);
    double2* gdiag = reinterpret_cast<double2*>(jac_raw + S::off_diag);
    double* rowoff = reinterpret_cast<double*>(jac_raw + S::off_row);
    double* red = reinterpret_cast<double*>(jac_raw + S::off_red);
    int* conv = reinterpret_cast<int*>(jac_raw + S::off_conv);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int wg = warp / S::NWN, wn = warp % S::NWN;  // row group, n-tile
    const int w = blockIdx.y, q0 = blockIdx.x * kJacQ;
    const int nvalid = min(kJacQ, a.nq - q0);
    const double2* Gw = a.Gamma + (size_t)w * N * N;   // row i of B (without its diagonal term): Gw[i N + j]

    // ---- set-up: D = 1/χ₀ of the CTA's q (q fastest in memory), Γ's diagonal and off-diagonal row sums
    for (int e = tid; e < N * kJacQ; e += kJacThreads) {
        const int i = e / kJacQ, c = e - i * kJacQ;
        double2 d = dmk(1.0, 0.0);
        if (c < nvalid) d = cinv(a.chi0[(size_t)(q0 + c) + (size_t)a.nq * (i + (size_t)N * w)]);
        D[i * S::LDX + c] = d;
    }
    for (int i = warp; i < N; i += kJacWarps) {       // one warp per row, coalesced, fixed-order sum
        double s = 0.0;
        for (int j = lane; j < N; j += 32) {
            const double2 g = Gw[(size_t)i * N + j];
            if (j != i) s += fabs(g.x) + fabs(g.y);
        }
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) {
            rowoff[i] = s;
            gdiag[i] = Gw[(size_t)i * N + i];
        }
    }
    if (tid < kJacQ) conv[tid] = tid < nvalid ? 0 : 1;
    __syncthreads();
    // x = diag(B)^-1 1 (padding q: 0)
    for (int e = tid; e < N * kJacQ; e += kJacThreads) {
        const int i = e / kJacQ, c = e - i * kJacQ;
        X[i * S::LDX + c] = c < nvalid ? cinv(cadd(gdiag[i], D[i * S::LDX + c])) : dmk(0.0, 0.0);
    }

    // one tile of Γ: rows 0..N-1, columns [kJacKC t, kJacKC (t + 1)), as 16-byte copies; every call
    // commits one group (empty past the last tile), so group t is tile t in every sweep
    auto load_tile = [&](int t) {
        if (t < NT) {
            double2* dst = G + (size_t)(t % NBUF) * S::tile;
            for (int e = tid; e < N * kJacKC; e += kJacThreads) {
                const int i = e / kJacKC, c = e - i * kJacKC;
                jac_cp16(dst + jac_tile_idx(i, c), Gw + (size_t)i * N + kJacKC * t + c);
            }
        }
        jac_commit();
    };

    const int fr = lane >> 2, fc = lane & 3;           // fragment row / column of this lane
    const int qa = 8 * wn + 2 * fc;                    // this lane's q pair: qa, qa + 1
    int it = 0;
    for (;; ++it) {
        // ---- R = B x without the diagonal 1/χ₀ term, on the FP64 tensor path
        // K3: S1 = Σ Re·Re, S2 = Σ Im·Im, S3 = Σ (Re + Im)(Re + Im); otherwise S1 = Re, S2 = Im directly
        double s1[S::MTW][2], s2[S::MTW][2], s3[K3 ? S::MTW : 1][2];
#pragma unroll
        for (int m = 0; m < S::MTW; ++m) s1[m][0] = s1[m][1] = s2[m][0] = s2[m][1] = 0.0;
#pragma unroll
        for (int m = 0; m < (K3 ? S::MTW : 1); ++m) s3[m][0] = s3[m][1] = 0.0;
#pragma unroll
        for (int t = 0; t < NBUF - 1; ++t) load_tile(t);
        for (int t = 0; t < NT; ++t) {
            jac_wait<NBUF - 2>();                      // group t (tile t) complete
            __syncthreads();                           // tile t visible; tile t - 1's buffer free
            load_tile(t + NBUF - 1);                   // into tile t - 1's buffer
            const double2* Gt = G + (size_t)(t % NBUF) * S::tile;
#pragma unroll
            for (int kk = 0; kk < kJacKC; kk += 4) {
                const double2 b = X[(kJacKC * t + kk + fc) * S::LDX + 8 * wn + fr];
                double2 g[S::MTW];
#pragma unroll
                for (int m = 0; m < S::MTW; ++m) g[m] = Gt[jac_tile_idx(8 * (wg * S::MTW + m) + fr, kk + fc)];
                if constexpr (K3) {
                    const double bs = b.x + b.y;
#pragma unroll
                    for (int m = 0; m < S::MTW; ++m) {
                        mma_f64(s1[m], g[m].x, b.x);
                        mma_f64(s2[m], g[m].y, b.y);
                        mma_f64(s3[m], g[m].x + g[m].y, bs);
                    }
                } else {
                    // four real products, in two rounds so that no accumulator is used twice in a row
                    const double bn = -b.y;
#pragma unroll
                    for (int m = 0; m < S::MTW; ++m) {
                        mma_f64(s1[m], g[m].x, b.x);
                        mma_f64(s2[m], g[m].x, b.y);
                    }
#pragma unroll
                    for (int m = 0; m < S::MTW; ++m) {
                        mma_f64(s1[m], g[m].y, bn);
                        mma_f64(s2[m], g[m].y, b.x);
                    }
                }
            }
        }
        // ---- residual and correction at this lane's (row, q) entries; per q the maxima of |r|, |x| and
        // |dx| (dx = r / B_ii, the next correction), and at the first sweep the row norm of B_q and the
        // Jacobi contraction bound theta_q (both fixed per q)
        double res[2] = {0.0, 0.0}, xn[2] = {0.0, 0.0}, dn[2] = {0.0, 0.0}, rn[2] = {0.0, 0.0}, th[2] = {0.0, 0.0};
        double2 dv[S::MTW][2];
#pragma unroll
        for (int m = 0; m < S::MTW; ++m) {
            const int i = 8 * (wg * S::MTW + m) + fr;
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const int q = qa + c;
                const double2 x = X[i * S::LDX + q];
                const double2 d = D[i * S::LDX + q];
                const double2 bx = cmul(d, x);
                const double2 gx = K3 ? dmk(s1[m][c] - s2[m][c], s3[K3 ? m : 0][c] - s1[m][c] - s2[m][c])
                                      : dmk(s1[m][c], s2[m][c]);
                const double2 r = dmk(1.0 - gx.x - bx.x, -gx.y - bx.y);
                const double2 bii = cadd(gdiag[i], d);
                const double2 dx = cdiv(r, bii);
                dv[m][c] = dx;
                res[c] = fmax(res[c], fabs(r.x) + fabs(r.y));
                xn[c] = fmax(xn[c], fabs(x.x) + fabs(x.y));
                dn[c] = fmax(dn[c], fabs(dx.x) + fabs(dx.y));
                if (it == 0) {
                    const double bd = fabs(bii.x) + fabs(bii.y);
                    rn[c] = fmax(rn[c], rowoff[i] + bd);
                    // |z| <= |Re z| + |Im z| <= sqrt(2) |z|: an upper bound of sum_{j != i} |B_ij| / |B_ii|
                    th[c] = fmax(th[c], kSqrt2 * rowoff[i] / bd);
                }
            }
        }
#pragma unroll
        for (int o = 4; o < 32; o <<= 1)
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                res[c] = fmax(res[c], __shfl_xor_sync(0xffffffffu, res[c], o));
                xn[c] = fmax(xn[c], __shfl_xor_sync(0xffffffffu, xn[c], o));
                dn[c] = fmax(dn[c], __shfl_xor_sync(0xffffffffu, dn[c], o));
                if (it == 0) {
                    rn[c] = fmax(rn[c], __shfl_xor_sync(0xffffffffu, rn[c], o));
                    th[c] = fmax(th[c], __shfl_xor_sync(0xffffffffu, th[c], o));
                }
            }
        if (fr == 0) {
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                red[(0 * 3 + wg) * kJacQ + qa + c] = res[c];
                red[(1 * 3 + wg) * kJacQ + qa + c] = xn[c];
                red[(2 * 3 + wg) * kJacQ + qa + c] = dn[c];
                if (it == 0) {
                    red[(3 * 3 + wg) * kJacQ + qa + c] = rn[c];
                    red[(4 * 3 + wg) * kJacQ + qa + c] = th[c];
                }
            }
        }
        __syncthreads();
        if (tid < kJacQ && !conv[tid]) {
            double rs = 0.0, xs = 0.0, ds = 0.0, rw = 0.0, tq = 0.0;
            for (int g = 0; g < 3; ++g) {
                rs = fmax(rs, red[(0 * 3 + g) * kJacQ + tid]);
                xs = fmax(xs, red[(1 * 3 + g) * kJacQ + tid]);
                ds = fmax(ds, red[(2 * 3 + g) * kJacQ + tid]);
                rw = fmax(rw, red[(3 * 3 + g) * kJacQ + tid]);
                tq = fmax(tq, red[(4 * 3 + g) * kJacQ + tid]);
            }
            // converged: the backward error of the LU kernels, max |r| / (max row norm * max |x| + 1), at
            // most 1e-14, and a forward bound: with theta < 1 the Jacobi map contracts in the max norm,
            // so |x* - x| <= |dx| / (1 - theta) <= 1e-14 |x| (|x| >= (|Re| + |Im|) / sqrt(2))
            const bool back = rs / (rw * xs + 1.0) <= kIterTol;
            const bool fwd = tq < 1.0 && ds / (1.0 - tq) <= kIterTol * xs / kSqrt2;
            if (back && fwd) conv[tid] = 1;
        }
        __syncthreads();
        int all = 1;
        for (int c = 0; c < kJacQ; ++c) all &= conv[c];
        if (all || it >= a.max_sweeps) break;
        // ---- x += dx for the q still above the bounds
#pragma unroll
        for (int m = 0; m < S::MTW; ++m) {
            const int i = 8 * (wg * S::MTW + m) + fr;
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const int q = qa + c;
                if (!conv[q]) X[i * S::LDX + q] = cadd(X[i * S::LDX + q], dv[m][c]);
            }
        }
        __syncthreads();                               // the reads of conv above precede its next update
    }

    // ---- χ = Σ_i Re x_i / β² per q (fixed order: shuffles, then the three row groups), then γ
    double cs[2] = {0.0, 0.0};
#pragma unroll
    for (int m = 0; m < S::MTW; ++m) {
        const int i = 8 * (wg * S::MTW + m) + fr;
#pragma unroll
        for (int c = 0; c < 2; ++c) cs[c] += X[i * S::LDX + qa + c].x;
    }
#pragma unroll
    for (int o = 4; o < 32; o <<= 1)
#pragma unroll
        for (int c = 0; c < 2; ++c) cs[c] += __shfl_xor_sync(0xffffffffu, cs[c], o);
    __syncthreads();                                   // red is free
    if (fr == 0) {
#pragma unroll
        for (int c = 0; c < 2; ++c) red[wg * kJacQ + qa + c] = cs[c];
    }
    __syncthreads();
    double chi[2];
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        const int q = qa + c;
        chi[c] = (red[q] + red[kJacQ + q] + red[2 * kJacQ + q]) / (a.beta * a.beta);
    }
    if (tid < nvalid) {
        const int q = tid;
        const double x = (red[q] + red[kJacQ + q] + red[2 * kJacQ + q]) / (a.beta * a.beta);
        const size_t o = (size_t)(q0 + q) + (size_t)a.nq * w;
        a.chi[o] = x;
        const bool ok = conv[q] != 0;
        a.flags[o] = ok ? 0 : 1;
        if (!ok && a.fail_list) a.fail_list[atomicAdd(a.fail_count, 1)] = (int32_t)o;
    }
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        const int q = qa + c;
        if (q >= nvalid) continue;
        const double f = 1.0 + a.s * a.U * chi[c];
#pragma unroll
        for (int m = 0; m < S::MTW; ++m) {
            const int i = 8 * (wg * S::MTW + m) + fr;
            const size_t ci = (size_t)(q0 + q) + (size_t)a.nq * (i + (size_t)N * w);
            a.gam[ci] = cdiv(X[i * S::LDX + q], cscale(a.chi0[ci], f));
        }
    }
}

template <int N, int Q, int NBUF, bool K3>
int run_jacobi_impl(ldga_ctx* ctx, const BseArgs& a, const BseArgs* a_d) {
    using S = JacSmem<N, Q, NBUF>;
    auto kern = k_bse_jacobi<N, Q, NBUF, K3>;
    LDGA_CUDA(ctx, set_smem(ctx, kern, S::bytes));
    StageTimer st_(ctx, LDGA_STAGE_BSE);
    dim3 grid((a.nq + Q - 1) / Q, a.nw, a_d ? 2 : 1);
    kern<<<grid, S::THREADS, S::bytes, ctx->stream>>>(a, a_d ? *a_d : a);
    LDGA_LAUNCHED(ctx, "k_bse_jacobi");
    return LDGA_OK;
}

template <int N, int Q, int NBUF, bool K3>
int run_jacobi(ldga_ctx* ctx, const BseArgs& a) { return run_jacobi_impl<N, Q, NBUF, K3>(ctx, a, nullptr); }

template <int N, int Q, int NBUF, bool K3>
int run_jacobi_pair(ldga_ctx* ctx, const BseArgs& a_m, const BseArgs& a_d) {
    return run_jacobi_impl<N, Q, NBUF, K3>(ctx, a_m, &a_d);
}
