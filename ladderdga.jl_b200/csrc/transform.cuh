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

// Apply S to `np` vectors: in[p*NQ + q] (wedge-indexed).  `consume(p, q_wedge, value)` receives
// every output exactly once.  bufA holds the inputs and is overwritten (3D stage 2); bufB is scratch.
// All threads of the CTA must call this; it synchronises internally and on exit.
template <int DIM, int M, class Consumer>
__device__ void sym_transform(int np, double2* bufA, double2* bufB, const TMat<M>& T, Consumer&& consume) {
    using S = TransformSmem<DIM, M>;
    constexpr int P2 = S::P2;
    constexpr int NQ = S::NQ;
    const int tid = threadIdx.x, nth = blockDim.x;
    if constexpr (DIM == 2) {
        // stage x: W1[qx][b] = sum_a T[qx][a] f(a, b)
        for (int it = tid; it < np * M; it += nth) {
            const int p = it / M, b = it - p * M;
            double2 v[M];
#pragma unroll
            for (int a = 0; a < M; ++a) v[a] = bufA[p * NQ + sidx2(a, b)];
            double2* w = bufB + p * (M * M);
#pragma unroll
            for (int qx = 0; qx < M; ++qx) w[qx * M + b] = trow<M>(T, qx, v);
        }
        __syncthreads();
        // stage y: out(qx, qy) = sum_b T[qy][b] W1[qx][b], qy <= qx
        for (int it = tid; it < np * M; it += nth) {
            const int p = it / M, qx = it - p * M;
            double2 v[M];
            const double2* w = bufB + p * (M * M) + qx * M;
#pragma unroll
            for (int b = 0; b < M; ++b) v[b] = w[b];
#pragma unroll
            for (int qy = 0; qy < M; ++qy) {
                if (qy <= qx) consume(p, widx2(qx, qy), trow<M>(T, qy, v));
            }
        }
        __syncthreads();
    } else {
        // stage x: W1[qx][(b,c)] = sum_a T[qx][a] f(a, b, c) for b >= c
        for (int it = tid; it < np * P2; it += nth) {
            const int p = it / P2, j = it - p * P2;
            int b, c;
            decode_pair(j, b, c);
            double2 v[M];
#pragma unroll
            for (int a = 0; a < M; ++a) v[a] = bufA[p * NQ + sidx3(a, b, c)];
            double2* w = bufB + p * (M * P2);
#pragma unroll
            for (int qx = 0; qx < M; ++qx) w[qx * P2 + j] = trow<M>(T, qx, v);
        }
        __syncthreads();
        // stage y: W2[(qx,qy)][c] = sum_b T[qy][b] W1[qx][(b,c)], qy <= qx  (W1 symmetric in b,c)
        for (int it = tid; it < np * M * M; it += nth) {
            const int p = it / (M * M), r = it - p * (M * M);
            const int qx = r / M, c = r - qx * M;
            double2 v[M];
            const double2* w = bufB + p * (M * P2) + qx * P2;
#pragma unroll
            for (int b = 0; b < M; ++b) v[b] = w[sidx2(b, c)];
            double2* o = bufA + p * S::BUF_A;
#pragma unroll
            for (int qy = 0; qy < M; ++qy) {
                if (qy <= qx) o[widx2(qx, qy) * M + c] = trow<M>(T, qy, v);
            }
        }
        __syncthreads();
        // stage z: out(qx,qy,qz) = sum_c T[qz][c] W2[(qx,qy)][c], qz <= qy
        for (int it = tid; it < np * P2; it += nth) {
            const int p = it / P2, pq = it - p * P2;
            int qx, qy;
            decode_pair(pq, qx, qy);
            double2 v[M];
            const double2* w = bufA + p * S::BUF_A + pq * M;
#pragma unroll
            for (int c = 0; c < M; ++c) v[c] = w[c];
#pragma unroll
            for (int qz = 0; qz < M; ++qz) {
                if (qz <= qy) consume(p, widx3(qx, qy, qz), trow<M>(T, qz, v));
            }
        }
        __syncthreads();
    }
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
