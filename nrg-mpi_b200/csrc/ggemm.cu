// Grouped FP64 GEMM with gathered operands: one launch runs every (sector pair, matrix
// type, local operation) product of a phase.  It replaces the per-pair dgemm calls of
// invariantMatrixDGEMM.F90:300,316, invariantMatrixForSpectrumDGEMM.F90:296,312,
// reducedDensityMatrixDGEMM.F90:280,296 and module.F90:1100,1113, without building the
// reference's dense coefficient matrices: rows of the eigenvector blocks are gathered
// through index lists instead.
//
//   C(i,j) = alpha * sum_k A(i,k) B(k,j) + beta * C(i,j)
//   A(i,k) = A[ri(i)*a_si + ki(k)*a_sk]          ri = a_ri ? a_ri[i] : i, ki likewise
//   B(k,j) = B[ki(k)*b_sk + ji(j)*b_sj]          ki = b_ki ? b_ki[k] : k, ji likewise
//   C(i,j) = C[ci(i)*c_si + cj(j)*c_sj]          ci = c_ri ? c_ri[i] : i, cj likewise
//
// 64x64 output tiles, 128 threads (four warps of 32x32), FP64 tensor-core MMA
// (mma.sync m8n8k4 f64); k slabs of 16 staged in shared memory, the next slab's global
// loads held in registers while the current slab is multiplied.  Loads are coalesced
// along whichever index of each operand has unit stride.
#include "internal.hpp"

namespace nrg {
namespace {

constexpr int TM = 64, TN = 64, TK = 16, NT = 128;
constexpr int LDA = TM + 4, LDB = TN + 4;   // [k][i] and [k][j] rows, padded against bank conflicts

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

struct Slab {
    double a[(TM * TK) / NT], b[(TN * TK) / NT];
};

__device__ __forceinline__ void fetch_slab(const GemmProblem& P, int i0, int j0, int k0, Slab& r, bool a_kfast,
                                           bool b_kfast) {
    const int tid = threadIdx.x;
#pragma unroll
    for (int u = 0; u < (TM * TK) / NT; ++u) {
        const int e = tid + u * NT;
        int ii, kk;
        if (a_kfast) { kk = e % TK; ii = e / TK; } else { ii = e % TM; kk = e / TM; }
        const int gi = i0 + ii, gk = k0 + kk;
        double v = 0.0;
        if (gi < P.M && gk < P.K) {
            const long long ri = P.a_ri ? P.a_ri[gi] : gi;
            const long long ki = P.a_ki ? P.a_ki[gk] : gk;
            v = P.A[ri * P.a_si + ki * P.a_sk];
        }
        r.a[u] = v;
    }
#pragma unroll
    for (int u = 0; u < (TN * TK) / NT; ++u) {
        const int e = tid + u * NT;
        int jj, kk;
        if (b_kfast) { kk = e % TK; jj = e / TK; } else { jj = e % TN; kk = e / TN; }
        const int gj = j0 + jj, gk = k0 + kk;
        double v = 0.0;
        if (gj < P.N && gk < P.K) {
            const long long ki = P.b_ki ? P.b_ki[gk] : gk;
            const long long ji = P.b_ji ? P.b_ji[gj] : gj;
            v = P.B[ki * P.b_sk + ji * P.b_sj];
        }
        r.b[u] = v;
    }
}

__device__ __forceinline__ void store_slab(const Slab& r, double* As, double* Bs, bool a_kfast, bool b_kfast) {
    const int tid = threadIdx.x;
#pragma unroll
    for (int u = 0; u < (TM * TK) / NT; ++u) {
        const int e = tid + u * NT;
        int ii, kk;
        if (a_kfast) { kk = e % TK; ii = e / TK; } else { ii = e % TM; kk = e / TM; }
        As[kk * LDA + ii] = r.a[u];
    }
#pragma unroll
    for (int u = 0; u < (TN * TK) / NT; ++u) {
        const int e = tid + u * NT;
        int jj, kk;
        if (b_kfast) { kk = e % TK; jj = e / TK; } else { jj = e % TN; kk = e / TN; }
        Bs[kk * LDB + jj] = r.b[u];
    }
}

__global__ void __launch_bounds__(NT) k_ggemm(const GemmProblem* __restrict__ probs,
                                              const int* __restrict__ tilePrefix, int nprob) {
    __shared__ double As[2][TK * LDA];
    __shared__ double Bs[2][TK * LDB];
    const int bid = blockIdx.x;
    int lo = 0, hi = nprob - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (tilePrefix[mid] <= bid) lo = mid; else hi = mid - 1;
    }
    GemmProblem P = probs[lo];
    const int t = bid - tilePrefix[lo];
    const int tilesN = (P.N + TN - 1) / TN;
    const int i0 = (t / tilesN) * TM, j0 = (t % tilesN) * TN;
    if (P.dyn_nk) {
        const int v = *P.dyn_nk;
        P.N = min(P.N, v);
        P.K = v;
        if (j0 >= P.N) return;
    }
    const bool a_kfast = (P.a_sk == 1 && P.a_si != 1);
    const bool b_kfast = (P.b_sk == 1 && P.b_sj != 1);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wi = (warp >> 1) * 32, wj = (warp & 1) * 32;   // warp tile origin
    const int g = lane >> 2, q4 = lane & 3;
    double acc[4][4][2];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[r][c][0] = acc[r][c][1] = 0.0;
    const int nslab = (P.K + TK - 1) / TK;
    Slab reg;
    if (nslab > 0) {
        fetch_slab(P, i0, j0, 0, reg, a_kfast, b_kfast);
        store_slab(reg, As[0], Bs[0], a_kfast, b_kfast);
    }
    __syncthreads();
    for (int s = 0; s < nslab; ++s) {
        const int cur = s & 1;
        if (s + 1 < nslab) fetch_slab(P, i0, j0, (s + 1) * TK, reg, a_kfast, b_kfast);
        const double* as = As[cur];
        const double* bs = Bs[cur];
#pragma unroll
        for (int ks = 0; ks < TK; ks += 4) {
            double af[4], bf[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) af[r] = as[(ks + q4) * LDA + wi + r * 8 + g];
#pragma unroll
            for (int c = 0; c < 4; ++c) bf[c] = bs[(ks + q4) * LDB + wj + c * 8 + g];
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int c = 0; c < 4; ++c) dmma(acc[r][c][0], acc[r][c][1], af[r], bf[c]);
        }
        if (s + 1 < nslab) store_slab(reg, As[cur ^ 1], Bs[cur ^ 1], a_kfast, b_kfast);
        __syncthreads();
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int gi = i0 + wi + r * 8 + g;
        if (gi >= P.M) continue;
        const long long ci = P.c_ri ? P.c_ri[gi] : gi;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int gj = j0 + wj + c * 8 + 2 * q4 + h;
                if (gj >= P.N) continue;
                const long long cj = P.c_ji ? P.c_ji[gj] : gj;
                double* out = P.C + ci * P.c_si + cj * P.c_sj;
                const double v = P.alpha * acc[r][c][h];
                *out = (P.beta == 0.0) ? v : P.beta * *out + v;
            }
        }
    }
}

}  // namespace

int launch_ggemm(nrg_context* ctx, std::vector<GemmProblem>& probs, int scratch_slot) {
    // drop empty problems
    std::vector<GemmProblem> live;
    live.reserve(probs.size());
    for (auto& p : probs)
        if (p.M > 0 && p.N > 0 && p.K > 0) live.push_back(p);
    const int np = (int)live.size();
    if (np == 0) return NRG_OK;
    std::vector<int> prefix(np);
    long long total = 0;
    for (int i = 0; i < np; ++i) {
        live[i].tiles = ((live[i].M + TM - 1) / TM) * ((live[i].N + TN - 1) / TN);
        prefix[i] = (int)total;
        total += live[i].tiles;
    }
    if (total > 0x7fffffffLL) return NRG_ERR_TOO_LARGE;
    DevBuf& dp = ctx->scratch.b[scratch_slot];
    DevBuf& dq = ctx->scratch.b[scratch_slot + 1];
    NRG_TRY(dp.ensure(sizeof(GemmProblem) * np));
    NRG_TRY(dq.ensure(sizeof(int) * np));
    NRG_TRY(h2d_async(ctx, dp.p, live.data(), sizeof(GemmProblem) * np));
    NRG_TRY(h2d_async(ctx, dq.p, prefix.data(), sizeof(int) * np));
    k_ggemm<<<(unsigned)total, NT, 0, ctx->stream>>>(dp.as<GemmProblem>(), dq.as<int>(), np);
    ctx->launches++;
    NRG_CUDA_TRY(cudaGetLastError());
    return NRG_OK;
}

}  // namespace nrg
