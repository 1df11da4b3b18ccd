// In-block FP64 GEMM with element accessors (gathers), used inside the eigensolver where
// one CTA owns a whole sector.  Register tile 4x4 per thread; the block covers a
// (ROWS x 64) output tile per pass with ROWS = 4 * blockDim.x / 16.
#pragma once
#include <cuda_runtime.h>

namespace nrg {

// C(i,j) = alpha * sum_k A(i,k) B(k,j) + (beta == 0 ? 0 : beta * C(i,j))
// fa(i,k), fb(k,j) return values (caller guarantees in-range indices are asked for);
// fc(i,j) returns a reference.  smem must hold 16*(ROWS+1) + 16*(64+1) doubles.
template <class FA, class FB, class FC>
__device__ void cta_gemm(int M, int N, int K, double alpha, double beta, FA fa, FB fb, FC fc,
                         double* smem) {
    const int nthr = blockDim.x;
    const int tid = threadIdx.x;
    const int ROWS = 4 * (nthr / 16);          // 512 threads -> 128 rows
    const int LDA = ROWS + 1, LDB = 65;
    double* As = smem;                          // [16][LDA]
    double* Bs = smem + 16 * LDA;               // [16][LDB]
    const int tx = tid % 16, ty = tid / 16;
    for (int i0 = 0; i0 < M; i0 += ROWS) {
        for (int j0 = 0; j0 < N; j0 += 64) {
            double acc[4][4];
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[r][c] = 0.0;
            for (int k0 = 0; k0 < K; k0 += 16) {
                for (int e = tid; e < 16 * ROWS; e += nthr) {
                    int ii = e % ROWS, kk = e / ROWS;
                    int gi = i0 + ii, gk = k0 + kk;
                    As[kk * LDA + ii] = (gi < M && gk < K) ? fa(gi, gk) : 0.0;
                }
                for (int e = tid; e < 16 * 64; e += nthr) {
                    int jj = e % 64, kk = e / 64;
                    int gj = j0 + jj, gk = k0 + kk;
                    Bs[kk * LDB + jj] = (gj < N && gk < K) ? fb(gk, gj) : 0.0;
                }
                __syncthreads();
#pragma unroll 4
                for (int kk = 0; kk < 16; ++kk) {
                    double a[4], b[4];
#pragma unroll
                    for (int r = 0; r < 4; ++r) a[r] = As[kk * LDA + ty * 4 + r];
#pragma unroll
                    for (int c = 0; c < 4; ++c) b[c] = Bs[kk * LDB + tx + 16 * c];
#pragma unroll
                    for (int r = 0; r < 4; ++r)
#pragma unroll
                        for (int c = 0; c < 4; ++c) acc[r][c] = fma(a[r], b[c], acc[r][c]);
                }
                __syncthreads();
            }
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                int gi = i0 + ty * 4 + r;
                if (gi >= M) continue;
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    int gj = j0 + tx + 16 * c;
                    if (gj >= N) continue;
                    double& out = fc(gi, gj);
                    out = (beta == 0.0) ? alpha * acc[r][c] : beta * out + alpha * acc[r][c];
                }
            }
        }
    }
}

}  // namespace nrg
