// Symmetry-reduced k-space transform S on the irreducible wedge, computed by one CTA for a batch of
// independent vectors held in shared memory.
//
// For f even in every axis and symmetric under axis permutations (all G, K and products of them
// in the ladder path are: they live on the point-group-reduced grid and are expanded from it),
//     S(f)(q) = sum_{R in full grid} f(R) exp(-2 pi i q.R/N) = sum_{R in [0,N/2]^d} prod_a T[q_a][R_a] f(R),
// and S(f) is again such a function, so only wedge inputs and wedge outputs are needed.  The sum is
// evaluated axis by axis (x, then y, then z), keeping after each stage only the index ranges later
// stages read: per vector 3D costs ~ M^4 + M^4 + Nq*M multiply-adds (M = N/2+1) instead of the
// full-grid FFT's N^3 log N, and no data ever leaves shared memory between stages.
//
// The convolution theorem used by the reference's conv_fft! / conv_tmp_add! then reads
//     (1/N_k) sum_k A(k) B(k+q) = S(S(A) S(B))(q) / N_k^2.
#pragma once

#include "ldga_internal.cuh"

namespace ldga {

__device__ __forceinline__ void decode_pair(int j, int& b, int& c) {
    int bb = (int)((sqrtf(8.0f * (float)j + 1.0f) - 1.0f) * 0.5f);
    while (bb * (bb + 1) / 2 > j) --bb;
    while ((bb + 1) * (bb + 2) / 2 <= j) ++bb;
    b = bb;
    c = j - bb * (bb + 1) / 2;
}

// Shared-memory words (double2) needed per vector: input/stage-2 buffer and stage-1 buffer.
template <int DIM, int M>
struct TransformSmem {
    static constexpr int P2 = M * (M + 1) / 2;
    static constexpr int NQ = DIM == 2 ? P2 : M * (M + 1) * (M + 2) / 6;
    static constexpr int BUF_A = DIM == 2 ? NQ : (NQ > P2 * M ? NQ : P2 * M);   // in, then stage-2
    static constexpr int BUF_B = DIM == 2 ? M * M : M * P2;                     // stage-1
};

// Dot product of one row of T (compile-time row/offsets when fully unrolled) with v.
template <int M>
__device__ __forceinline__ double2 trow(const TMat<M>& T, int row, const double2 (&v)[M]) {
    double re = 0.0, im = 0.0;
#pragma unroll
    for (int a = 0; a < M; ++a) {
        const double t = T.t[row * M + a];
        re = fma(t, v[a].x, re);
        im = fma(t, v[a].y, im);
    }
    return make_double2(re, im);
}

// Output rows of a stage are split into RS chunks so that each stage has enough independent work
// items for the CTA (a stage has only M, P2 or M^2 columns per vector).  A chunk is a compile-time
// row range, so every T coefficient stays an immediate constant-bank operand of its FMA; the items of
// one chunk are padded to whole warps, so every warp applies one chunk.
template <int DIM, int M>
struct RowSplit {
    static constexpr int RS = M >= 17 ? (DIM == 2 ? 4 : 2) : (M >= 9 ? 2 : 1);
    static constexpr int CH = (M + RS - 1) / RS;
};

// rows r = C CH .. C CH + CH - 1 (r < M, r <= lim) of T v, each handed to f(r, value)
template <int M, int CH, int C, class F>
__device__ __forceinline__ void rows_chunk(const TMat<M>& T, const double2 (&v)[M], int lim, F&& f) {
#pragma unroll
    for (int qq = 0; qq < CH; ++qq) {
        const int r = C * CH + qq;
        if (r < M && r <= lim) f(r, trow<M>(T, r, v));
    }
}

template <int DIM, int M, class F>
__device__ __forceinline__ void rows_of(int chunk, const TMat<M>& T, const double2 (&v)[M], int lim, F&& f) {
    using R = RowSplit<DIM, M>;
    if (chunk == 0) rows_chunk<M, R::CH, 0>(T, v, lim, f);
    if constexpr (R::RS > 1) { if (chunk == 1) rows_chunk<M, R::CH, 1>(T, v, lim, f); }
    if constexpr (R::RS > 2) { if (chunk == 2) rows_chunk<M, R::CH, 2>(T, v, lim, f); }
    if constexpr (R::RS > 3) { if (chunk == 3) rows_chunk<M, R::CH, 3>(T, v, lim, f); }
}

// for it in [0, RS * IPC): chunk = it / IPC, local item = it % IPC (< n), IPC = n rounded up to 32
template <int DIM, int M, class Body>
__device__ __forceinline__ void for_items(int n, Body&& body) {
    using R = RowSplit<DIM, M>;
    const int ipc = (n + 31) & ~31;
    for (int it = threadIdx.x; it < R::RS * ipc; it += blockDim.x) {
        const int chunk = it / ipc, loc = it - chunk * ipc;
        if (loc < n) body(chunk, loc);
    }
}

// Apply S to `np` vectors: in[p*NQ + q] (wedge-indexed).  `consume(p, q_wedge, value)` receives
// every output exactly once.  bufA holds the inputs and is overwritten (3D stage 2); bufB is scratch.
// All threads of the CTA must call this; it synchronises internally and on exit.
template <int DIM, int M, class Consumer>
__device__ void sym_transform(int np, double2* bufA, double2* bufB, const TMat<M>& T, Consumer&& consume) {
    using S = TransformSmem<DIM, M>;
    constexpr int P2 = S::P2;
    constexpr int NQ = S::NQ;
    if constexpr (DIM == 2) {
        // stage x: W1[qx][b] = sum_a T[qx][a] f(a, b)
        for_items<DIM, M>(np * M, [&](int chunk, int it) {
            const int p = it / M, b = it - p * M;
            double2 v[M];
#pragma unroll
            for (int a = 0; a < M; ++a) v[a] = bufA[p * NQ + sidx2(a, b)];
            double2* w = bufB + p * (M * M);
            rows_of<DIM, M>(chunk, T, v, M - 1, [&](int qx, double2 y) { w[qx * M + b] = y; });
        });
        __syncthreads();
        // stage y: out(qx, qy) = sum_b T[qy][b] W1[qx][b], qy <= qx
        for_items<DIM, M>(np * M, [&](int chunk, int it) {
            const int p = it / M, qx = it - p * M;
            if (chunk * RowSplit<DIM, M>::CH > qx) return;
            double2 v[M];
            const double2* w = bufB + p * (M * M) + qx * M;
#pragma unroll
            for (int b = 0; b < M; ++b) v[b] = w[b];
            rows_of<DIM, M>(chunk, T, v, qx, [&](int qy, double2 y) { consume(p, widx2(qx, qy), y); });
        });
        __syncthreads();
    } else {
        // stage x: W1[qx][(b,c)] = sum_a T[qx][a] f(a, b, c) for b >= c
        for_items<DIM, M>(np * P2, [&](int chunk, int it) {
            const int p = it / P2, j = it - p * P2;
            int b, c;
            decode_pair(j, b, c);
            double2 v[M];
#pragma unroll
            for (int a = 0; a < M; ++a) v[a] = bufA[p * NQ + sidx3(a, b, c)];
            double2* w = bufB + p * (M * P2);
            rows_of<DIM, M>(chunk, T, v, M - 1, [&](int qx, double2 y) { w[qx * P2 + j] = y; });
        });
        __syncthreads();
        // stage y: W2[(qx,qy)][c] = sum_b T[qy][b] W1[qx][(b,c)], qy <= qx  (W1 symmetric in b,c)
        for_items<DIM, M>(np * M * M, [&](int chunk, int it) {
            const int p = it / (M * M), r = it - p * (M * M);
            const int qx = r / M, c = r - qx * M;
            if (chunk * RowSplit<DIM, M>::CH > qx) return;
            double2 v[M];
            const double2* w = bufB + p * (M * P2) + qx * P2;
#pragma unroll
            for (int b = 0; b < M; ++b) v[b] = w[sidx2(b, c)];
            double2* o = bufA + p * S::BUF_A;
            rows_of<DIM, M>(chunk, T, v, qx, [&](int qy, double2 y) { o[widx2(qx, qy) * M + c] = y; });
        });
        __syncthreads();
        // stage z: out(qx,qy,qz) = sum_c T[qz][c] W2[(qx,qy)][c], qz <= qy
        for_items<DIM, M>(np * P2, [&](int chunk, int it) {
            const int p = it / P2, pq = it - p * P2;
            int qx, qy;
            decode_pair(pq, qx, qy);
            if (chunk * RowSplit<DIM, M>::CH > qy) return;
            double2 v[M];
            const double2* w = bufA + p * S::BUF_A + pq * M;
#pragma unroll
            for (int c = 0; c < M; ++c) v[c] = w[c];
            rows_of<DIM, M>(chunk, T, v, qy, [&](int qz, double2 y) { consume(p, widx3(qx, qy, qz), y); });
        });
        __syncthreads();
    }
}

// ------------------------------------------------------------------------------------------------
// The same transform on the FP64 tensor path.  Every stage is T times a set of columns, T fixed: with
// mma.sync.m8n8k4 (FP64 operands, FP64 accumulation) T is the A operand, kept in registers as
// fragments of its 8 x 4 tiles (rows and k padded with zeros to multiples of 8 and 4), and the
// columns -- real and imaginary parts of 4 complex columns per 8-column tile -- are the B operand,
// gathered from shared memory (lane l holds B[k = l % 4][n = l / 4], n = 2 j + part of complex column
// j).  The accumulator gives lane l the complex output of row l / 4, column l % 4 (C[g][2t], C[g][2t+1]
// are its real and imaginary parts).  Warps take 8-column tiles in turn; a tile computes only the
// row tiles its columns need (stage y: qy <= qx, stage z: qz <= qy).  One tensor instruction replaces
// 256 FP64 FMAs, and no thread holds a column in registers (the CUDA-core form keeps M complex values
// per thread), so the kernels need far fewer registers.
template <int M>
struct TFrag {
    static constexpr int RT = (M + 7) / 8, KT = (M + 3) / 4;
    double a[RT][KT];
};

__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

template <int M>
__device__ __forceinline__ void load_tfrag(const TMat<M>& T, TFrag<M>& F, int lane) {
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int rt = 0; rt < TFrag<M>::RT; ++rt)
#pragma unroll
        for (int kt = 0; kt < TFrag<M>::KT; ++kt) {
            const int r = rt * 8 + g, k = kt * 4 + t;
            F.a[rt][kt] = (r < M && k < M) ? T.t[r * M + k] : 0.0;
        }
}

// One stage over `ncol` complex columns.  colB(j, k) returns column j's k-th input (k < M, j < ncol);
// rows(j) the largest output row column j needs (< M); out(j, r, v) receives row r of column j for every
// r <= rows(j).
template <int M, class ColB, class Rows, class Out>
__device__ __forceinline__ void tc_stage(const TFrag<M>& F, int ncol, ColB&& colB, Rows&& rows, Out&& out) {
    constexpr int RT = TFrag<M>::RT, KT = TFrag<M>::KT;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int ntile = (ncol + 3) / 4;
    for (int ct = warp; ct < ntile; ct += nwarp) {
        const int jb = ct * 4 + (g >> 1), part = g & 1;
        double b[KT];
#pragma unroll
        for (int kt = 0; kt < KT; ++kt) {
            const int k = kt * 4 + t;
            double v = 0.0;
            if (jb < ncol && k < M) {
                const double2 z = colB(jb, k);
                v = part ? z.y : z.x;
            }
            b[kt] = v;
        }
        int rmax = -1;
#pragma unroll
        for (int c = 0; c < 4; ++c)
            if (ct * 4 + c < ncol) rmax = max(rmax, rows(ct * 4 + c));
        const int jo = ct * 4 + t;
        // the row tiles' accumulations are independent chains: interleaved over k so that consecutive
        // tensor instructions do not wait for each other (the row-tile guard is uniform over the warp)
        double acc[RT][2];
#pragma unroll
        for (int rt = 0; rt < RT; ++rt) acc[rt][0] = acc[rt][1] = 0.0;
#pragma unroll
        for (int kt = 0; kt < KT; ++kt)
#pragma unroll
            for (int rt = 0; rt < RT; ++rt)
                if (rt * 8 <= rmax) dmma(acc[rt], F.a[rt][kt], b[kt]);
#pragma unroll
        for (int rt = 0; rt < RT; ++rt) {
            const int r = rt * 8 + g;
            if (rt * 8 <= rmax && jo < ncol && r <= rows(jo)) out(jo, r, make_double2(acc[rt][0], acc[rt][1]));
        }
    }
}

// sym_transform's interface and buffers on the tensor path.
template <int DIM, int M, class Consumer>
__device__ void sym_transform_tc(int np, double2* bufA, double2* bufB, const TMat<M>& T, Consumer&& consume) {
    using S = TransformSmem<DIM, M>;
    constexpr int P2 = S::P2;
    constexpr int NQ = S::NQ;
    TFrag<M> F;
    load_tfrag<M>(T, F, threadIdx.x & 31);
    if constexpr (DIM == 2) {
        // stage x: W1[qx][b] = sum_a T[qx][a] f(a, b); column j = (p, b)
        tc_stage<M>(F, np * M,
            [&](int j, int k) { const int p = j / M, b = j - p * M; return bufA[p * NQ + sidx2(k, b)]; },
            [&](int) { return M - 1; },
            [&](int j, int r, double2 v) { const int p = j / M, b = j - p * M; bufB[p * (M * M) + r * M + b] = v; });
        __syncthreads();
        // stage y: out(qx, qy) = sum_b T[qy][b] W1[qx][b], qy <= qx; column j = (p, qx)
        tc_stage<M>(F, np * M,
            [&](int j, int k) { const int p = j / M, qx = j - p * M; return bufB[p * (M * M) + qx * M + k]; },
            [&](int j) { return j % M; },
            [&](int j, int r, double2 v) { const int p = j / M, qx = j - p * M; consume(p, widx2(qx, r), v); });
        __syncthreads();
    } else {
        // stage x: W1[qx][(b, c)] = sum_a T[qx][a] f(a, b, c), b >= c; column j = (p, pair)
        tc_stage<M>(F, np * P2,
            [&](int j, int k) {
                const int p = j / P2, pr = j - p * P2;
                int b, c;
                decode_pair(pr, b, c);
                return bufA[p * NQ + sidx3(k, b, c)];
            },
            [&](int) { return M - 1; },
            [&](int j, int r, double2 v) { const int p = j / P2, pr = j - p * P2; bufB[p * (M * P2) + r * P2 + pr] = v; });
        __syncthreads();
        // stage y: W2[(qx, qy)][c] = sum_b T[qy][b] W1[qx][(b, c)], qy <= qx; column j = (p, qx, c)
        tc_stage<M>(F, np * M * M,
            [&](int j, int k) {
                const int p = j / (M * M), rr = j - p * (M * M), qx = rr / M, c = rr - qx * M;
                return bufB[p * (M * P2) + qx * P2 + sidx2(k, c)];
            },
            [&](int j) { return (j % (M * M)) / M; },
            [&](int j, int r, double2 v) {
                const int p = j / (M * M), rr = j - p * (M * M), qx = rr / M, c = rr - qx * M;
                bufA[p * S::BUF_A + widx2(qx, r) * M + c] = v;
            });
        __syncthreads();
        // stage z: out(qx, qy, qz) = sum_c T[qz][c] W2[(qx, qy)][c], qz <= qy; column j = (p, pair)
        tc_stage<M>(F, np * P2,
            [&](int j, int k) { const int p = j / P2, pq = j - p * P2; return bufA[p * S::BUF_A + pq * M + k]; },
            [&](int j) {
                int qx, qy;
                decode_pair(j % P2, qx, qy);
                return qy;
            },
            [&](int j, int r, double2 v) {
                const int p = j / P2, pq = j - p * P2;
                int qx, qy;
                decode_pair(pq, qx, qy);
                consume(p, widx3(qx, qy, r), v);
            });
        __syncthreads();
    }
}

// the CUDA-core or the tensor-path form, chosen at compile time
template <int DIM, int M, bool TC, class Consumer>
__device__ __forceinline__ void sym_transform_any(int np, double2* bufA, double2* bufB, const TMat<M>& T,
                                                  Consumer&& consume) {
    if constexpr (TC) sym_transform_tc<DIM, M>(np, bufA, bufB, T, consume);
    else sym_transform<DIM, M>(np, bufA, bufB, T, consume);
}

}  // namespace ldga

// Instantiation list: (DIM, M) pairs the library is built for.  M = N/2 + 1.
//   N = 1 (one-point grid of the local quantities) in 2D and 3D
//   2D: N = 2, 4, 6, 8, 10, 12, 16, 20, 24, 32, 40, 48, 64
//   3D: N = 2, 4, 6, 8, 10, 12, 16, 20, 24, 32
#define LDGA_FOR_EACH_GRID(X)                                                              \
    X(2, 1) X(3, 1) X(2, 2) X(2, 3) X(2, 4) X(2, 5) X(2, 6) X(2, 7) X(2, 9) X(2, 11) X(2, 13) X(2, 17)      \
    X(2, 21) X(2, 25) X(2, 33)                                                             \
    X(3, 2) X(3, 3) X(3, 4) X(3, 5) X(3, 6) X(3, 7) X(3, 9) X(3, 11) X(3, 13) X(3, 17)
