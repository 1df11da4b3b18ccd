// In-block FP64 GEMM with element accessors (gathers), used inside the eigensolver where
// one CTA of 512 threads owns a whole sector or merge.  FP64 tensor-core MMA
// (mma.sync m8n8k4 f64): the block covers a 128 x 64 output tile per pass, sixteen warps
// of 32 x 16 (four by two 8 x 8 MMA tiles each); k slabs of 16 are staged in shared
// memory, the next slab's loads held in registers while the current one is multiplied.
#pragma once
#include <cuda_runtime.h>

namespace nrg {

constexpr int kCtaThreads = 512;                       // the only block size the GEMM is written for
constexpr int kCtaRows = 128, kCtaCols = 64, kCtaK = 16;
constexpr int kCtaLdA = kCtaRows + 4, kCtaLdB = kCtaCols + 4;   // = 4 mod 16: conflict-free fragments
constexpr int kCtaGemmSmem = kCtaK * kCtaLdA + kCtaK * kCtaLdB;  // doubles of staging

__device__ __forceinline__ void cta_dmma(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// C(i,j) = alpha * sum_k A(i,k) B(k,j) + (beta == 0 ? 0 : beta * C(i,j))
// fa(i,k), fb(k,j) return values (only in-range indices are asked for); fc(i,j) returns a
// reference.  smem holds kCtaGemmSmem doubles.  Every thread of the block calls it.
template <class FA, class FB, class FC>
__device__ void cta_gemm(int M, int N, int K, double alpha, double beta, FA fa, FB fb, FC fc,
                         double* smem) {
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int wi = (warp >> 2) * 32, wj = (warp & 3) * 16;   // warp tile origin
    const int g = lane >> 2, q4 = lane & 3;
    double* As = smem;                       // [k][i], leading dim kCtaLdA
    double* Bs = smem + kCtaK * kCtaLdA;     // [k][j], leading dim kCtaLdB
    constexpr int NA = kCtaRows * kCtaK / kCtaThreads, NBv = kCtaCols * kCtaK / kCtaThreads;
    for (int i0 = 0; i0 < M; i0 += kCtaRows) {
        for (int j0 = 0; j0 < N; j0 += kCtaCols) {
            double acc[4][2][2];
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int c = 0; c < 2; ++c) acc[r][c][0] = acc[r][c][1] = 0.0;
            double ra[NA], rb[NBv];
            auto fetch = [&](int k0) {
#pragma unroll
                for (int u = 0; u < NA; ++u) {
                    const int e = tid + u * kCtaThreads, ii = e % kCtaRows, kk = e / kCtaRows;
                    const int gi = i0 + ii, gk = k0 + kk;
                    ra[u] = (gi < M && gk < K) ? fa(gi, gk) : 0.0;
                }
#pragma unroll
                for (int u = 0; u < NBv; ++u) {
                    const int e = tid + u * kCtaThreads, jj = e % kCtaCols, kk = e / kCtaCols;
                    const int gj = j0 + jj, gk = k0 + kk;
                    rb[u] = (gj < N && gk < K) ? fb(gk, gj) : 0.0;
                }
            };
            auto store = [&]() {
#pragma unroll
                for (int u = 0; u < NA; ++u) {
                    const int e = tid + u * kCtaThreads;
                    As[(e / kCtaRows) * kCtaLdA + e % kCtaRows] = ra[u];
                }
#pragma unroll
                for (int u = 0; u < NBv; ++u) {
                    const int e = tid + u * kCtaThreads;
                    Bs[(e / kCtaCols) * kCtaLdB + e % kCtaCols] = rb[u];
                }
            };
            fetch(0);
            for (int k0 = 0; k0 < K; k0 += kCtaK) {
                __syncthreads();   // the previous slab is no longer read
                store();
                __syncthreads();
                if (k0 + kCtaK < K) fetch(k0 + kCtaK);
#pragma unroll
                for (int ks = 0; ks < kCtaK; ks += 4) {
                    double af[4], bf[2];
#pragma unroll
                    for (int r = 0; r < 4; ++r) af[r] = As[(ks + q4) * kCtaLdA + wi + r * 8 + g];
#pragma unroll
                    for (int c = 0; c < 2; ++c) bf[c] = Bs[(ks + q4) * kCtaLdB + wj + c * 8 + g];
#pragma unroll
                    for (int r = 0; r < 4; ++r)
#pragma unroll
                        for (int c = 0; c < 2; ++c) cta_dmma(acc[r][c][0], acc[r][c][1], af[r], bf[c]);
                }
            }
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int gi = i0 + wi + r * 8 + g;
                if (gi >= M) continue;
#pragma unroll
                for (int c = 0; c < 2; ++c)
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int gj = j0 + wj + c * 8 + 2 * q4 + h;
                        if (gj >= N) continue;
                        double& out = fc(gi, gj);
                        out = (beta == 0.0) ? alpha * acc[r][c][h] : beta * out + alpha * acc[r][c][h];
                    }
            }
            __syncthreads();   // staging is reused by the next tile or the caller
        }
    }
}

}  // namespace nrg
