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
// Output tiles of 32x32 per warp (64x64 with four warps, 32x32 with one, 128x64 and
// 64x128 with eight), FP64 tensor-core MMA (mma.sync m8n8k4 f64); k slabs of 16 staged in
// shared memory, the next slab's global loads held in registers while the current slab is
// multiplied.  Loads are coalesced along whichever index of each operand has unit stride.
// The tile shape of each launch is chosen by the context's tuner (GemmTuner below).
#include "internal.hpp"

#include <algorithm>
#include <cstdlib>
#include <map>
#include <mutex>

namespace nrg {
namespace {

constexpr int TK = 16;

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// WM x WN warps per block, each computing a 32 x 32 piece of the (32 WM) x (32 WN) output
// tile.  Every variant accumulates each output element over k in the same order (slabs of
// 16, then the k = 4 steps of the MMA), so all variants give bit-identical results and the
// tile choice is free to change between launches.
template <int WM, int WN>
struct Tile {
    static constexpr int TM = 32 * WM, TN = 32 * WN, NT = 32 * WM * WN;
    static constexpr int LDA = TM + 4, LDB = TN + 4;   // [k][i] and [k][j] rows, padded
    static constexpr int EA = (TM * TK) / NT, EB = (TN * TK) / NT;
    static constexpr size_t smem_bytes() { return sizeof(double) * 2 * TK * (LDA + LDB); }
};

template <class T>
struct Slab {
    double a[T::EA], b[T::EB];
};

template <class T>
__device__ __forceinline__ void fetch_slab(const GemmProblem& P, int i0, int j0, int k0, Slab<T>& r, bool a_kfast,
                                           bool b_kfast) {
    const int tid = threadIdx.x;
#pragma unroll
    for (int u = 0; u < T::EA; ++u) {
        const int e = tid + u * T::NT;
        int ii, kk;
        if (a_kfast) { kk = e % TK; ii = e / TK; } else { ii = e % T::TM; kk = e / T::TM; }
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
    for (int u = 0; u < T::EB; ++u) {
        const int e = tid + u * T::NT;
        int jj, kk;
        if (b_kfast) { kk = e % TK; jj = e / TK; } else { jj = e % T::TN; kk = e / T::TN; }
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

template <class T>
__device__ __forceinline__ void store_slab(const Slab<T>& r, double* As, double* Bs, bool a_kfast, bool b_kfast) {
    const int tid = threadIdx.x;
#pragma unroll
    for (int u = 0; u < T::EA; ++u) {
        const int e = tid + u * T::NT;
        int ii, kk;
        if (a_kfast) { kk = e % TK; ii = e / TK; } else { ii = e % T::TM; kk = e / T::TM; }
        As[kk * T::LDA + ii] = r.a[u];
    }
#pragma unroll
    for (int u = 0; u < T::EB; ++u) {
        const int e = tid + u * T::NT;
        int jj, kk;
        if (b_kfast) { kk = e % TK; jj = e / TK; } else { jj = e % T::TN; kk = e / T::TN; }
        Bs[kk * T::LDB + jj] = r.b[u];
    }
}

template <int WM, int WN>
__global__ void __launch_bounds__(32 * WM * WN) k_ggemm(const GemmProblem* __restrict__ probs,
                                                        const int* __restrict__ tilePrefix, int nprob) {
    using T = Tile<WM, WN>;
    extern __shared__ double gsm[];
    // two A slabs, then two B slabs
    auto As = [&](int x) { return gsm + x * (TK * T::LDA); };
    auto Bs = [&](int x) { return gsm + 2 * TK * T::LDA + x * (TK * T::LDB); };
    const int bid = blockIdx.x;
    int lo = 0, hi = nprob - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (tilePrefix[mid] <= bid) lo = mid; else hi = mid - 1;
    }
    GemmProblem P = probs[lo];
    const int t = bid - tilePrefix[lo];
    const int tilesN = (P.N + T::TN - 1) / T::TN;
    const int i0 = (t / tilesN) * T::TM, j0 = (t % tilesN) * T::TN;
    if (P.dyn_nk) {
        const int v = *P.dyn_nk;
        P.N = min(P.N, v);
        P.K = v;
        if (j0 >= P.N) return;
    }
    const bool a_kfast = (P.a_sk == 1 && P.a_si != 1);
    const bool b_kfast = (P.b_sk == 1 && P.b_sj != 1);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wi = (warp / WN) * 32, wj = (warp % WN) * 32;   // warp tile origin
    const int g = lane >> 2, q4 = lane & 3;
    double acc[4][4][2];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[r][c][0] = acc[r][c][1] = 0.0;
    const int nslab = (P.K + TK - 1) / TK;
    Slab<T> reg;
    if (nslab > 0) {
        fetch_slab<T>(P, i0, j0, 0, reg, a_kfast, b_kfast);
        store_slab<T>(reg, As(0), Bs(0), a_kfast, b_kfast);
    }
    __syncthreads();
    for (int s = 0; s < nslab; ++s) {
        const int cur = s & 1;
        if (s + 1 < nslab) fetch_slab<T>(P, i0, j0, (s + 1) * TK, reg, a_kfast, b_kfast);
        const double* as = As(cur);
        const double* bs = Bs(cur);
#pragma unroll
        for (int ks = 0; ks < TK; ks += 4) {
            double af[4], bf[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) af[r] = as[(ks + q4) * T::LDA + wi + r * 8 + g];
#pragma unroll
            for (int c = 0; c < 4; ++c) bf[c] = bs[(ks + q4) * T::LDB + wj + c * 8 + g];
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int c = 0; c < 4; ++c) dmma(acc[r][c][0], acc[r][c][1], af[r], bf[c]);
        }
        if (s + 1 < nslab) store_slab<T>(reg, As(cur ^ 1), Bs(cur ^ 1), a_kfast, b_kfast);
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

// the tile variants, in the order of GemmTuner's slots
constexpr int kVariants = 4;
constexpr int kWM[kVariants] = {2, 1, 4, 2};
constexpr int kWN[kVariants] = {2, 1, 2, 4};

template <int WM, int WN>
int launch_variant(nrg_context* ctx, long long total_blocks_hint, const GemmProblem* dp, const int* dq, int np,
                   const std::vector<GemmProblem>& live, std::vector<int>& prefix, DevBuf& prefixBuf) {
    using T = Tile<WM, WN>;
    long long total = 0;
    for (int i = 0; i < np; ++i) {
        prefix[i] = (int)total;
        total += (long long)((live[i].M + T::TM - 1) / T::TM) * ((live[i].N + T::TN - 1) / T::TN);
    }
    (void)total_blocks_hint;
    if (total > 0x7fffffffLL) return NRG_ERR_TOO_LARGE;
    NRG_TRY(h2d_async(ctx, prefixBuf.p, prefix.data(), sizeof(int) * np));
    const size_t smem = T::smem_bytes();
    if (smem > 48 * 1024) NRG_TRY(raise_smem_limit((const void*)k_ggemm<WM, WN>, smem));
    k_ggemm<WM, WN><<<(unsigned)total, T::NT, smem, ctx->stream>>>(dp, dq, np);
    ctx->launches++;
    NRG_CUDA_TRY(cudaGetLastError());
    return NRG_OK;
}

int log2_bucket(long long v) {
    int b = 0;
    while (v > 1 && b < 15) { v >>= 1; ++b; }
    return b;
}

}  // namespace

// Online tuning of the tile shape, per device.  Launches are keyed by their problem mix
// (log2 buckets of the median M, N, K and of the problem count); the first launches of a
// key try each tile variant in turn, timed by events on the launching stream, and later
// launches of the key take the variant with the least time per flop.  Timings are read without
// waiting: a pending measurement is collected by a later launch once its events have
// completed.  The variants give bit-identical results, so the choice never changes a
// result.  NRG_GGEMM_VARIANT=0..3 fixes one variant (no tuning).
int GemmTuner::pick(unsigned key) {
    static const int forced = [] {
        const char* e = getenv("NRG_GGEMM_VARIANT");
        if (!e || !*e) return -1;
        const int v = atoi(e);
        return (v >= 0 && v < kTunedVariants) ? v : -1;
    }();
    if (forced >= 0) return forced;
    Entry& e = table[key];
    for (int v = 0; v < kTunedVariants; ++v)
        if (e.samples[v] < kSamples && e.inflight[v] == 0) return v;
    int best = 0;
    for (int v = 1; v < kTunedVariants; ++v)
        if (e.samples[v] > 0 && (e.samples[best] == 0 || e.ms_per_gflop[v] < e.ms_per_gflop[best])) best = v;
    return best;
}

void GemmTuner::collect(bool wait) {
    for (size_t i = 0; i < pending.size();) {
        Pending& q = pending[i];
        cudaError_t st = wait ? cudaEventSynchronize(q.b) : cudaEventQuery(q.b);
        if (st == cudaErrorNotReady) { ++i; continue; }
        float ms = 0.0f;
        if (st == cudaSuccess && cudaEventElapsedTime(&ms, q.a, q.b) == cudaSuccess && q.gflop > 0.0) {
            Entry& e = table[q.key];
            const double r = ms / q.gflop;
            e.ms_per_gflop[q.variant] = e.samples[q.variant] == 0 ? r : std::min(e.ms_per_gflop[q.variant], r);
            e.samples[q.variant]++;
            e.inflight[q.variant]--;
        } else {
            cudaGetLastError();
            table[q.key].inflight[q.variant]--;
        }
        free_events.push_back(q.a);
        free_events.push_back(q.b);
        pending[i] = pending.back();
        pending.pop_back();
    }
}

// one tuner per device, shared by every context on it (independent instances side by side
// tune once between them); its state is guarded by its mutex
GemmTuner& tuner_for(int dev) {
    static std::mutex mu;
    static std::map<int, GemmTuner*> tuners;
    std::lock_guard<std::mutex> lk(mu);
    GemmTuner*& t = tuners[dev];
    if (!t) t = new GemmTuner();   // lives until the process exits
    return *t;
}

int launch_ggemm(nrg_context* ctx, std::vector<GemmProblem>& probs, int scratch_slot) {
    // drop empty problems
    std::vector<GemmProblem> live;
    live.reserve(probs.size());
    for (auto& p : probs)
        if (p.M > 0 && p.N > 0 && p.K > 0) live.push_back(p);
    const int np = (int)live.size();
    if (np == 0) return NRG_OK;
    // problem-mix key and algorithmic flops
    std::vector<int> ms(np), ns(np), ks(np);
    double gflop = 0.0;
    for (int i = 0; i < np; ++i) {
        ms[i] = live[i].M;
        ns[i] = live[i].N;
        ks[i] = live[i].K;
        gflop += 2e-9 * live[i].M * (double)live[i].N * live[i].K;
    }
    auto med = [](std::vector<int>& v) {
        std::nth_element(v.begin(), v.begin() + v.size() / 2, v.end());
        return (long long)v[v.size() / 2];
    };
    const unsigned key = (unsigned)(log2_bucket(med(ms)) | log2_bucket(med(ns)) << 4 | log2_bucket(med(ks)) << 8 |
                                    log2_bucket(np) << 12);
    int dev = 0;
    NRG_CUDA_TRY(cudaGetDevice(&dev));
    GemmTuner& tu = tuner_for(dev);
    std::unique_lock<std::mutex> lk(tu.mu);
    tu.collect(false);
    const int v = tu.pick(key);
    DevBuf& dp = ctx->scratch.b[scratch_slot];
    DevBuf& dq = ctx->scratch.b[scratch_slot + 1];
    NRG_TRY(dp.ensure(sizeof(GemmProblem) * np));
    NRG_TRY(dq.ensure(sizeof(int) * np));
    for (auto& p : live) p.tiles = 0;   // unused by the kernels (the prefix carries the tiling)
    NRG_TRY(h2d_async(ctx, dp.p, live.data(), sizeof(GemmProblem) * np));
    std::vector<int> prefix(np);
    const bool timed = tu.table[key].samples[v] < GemmTuner::kSamples && tu.table[key].inflight[v] == 0;
    cudaEvent_t ea = nullptr, eb = nullptr;
    if (timed) {
        NRG_TRY(tu.event(&ea));
        NRG_TRY(tu.event(&eb));
        tu.table[key].inflight[v]++;   // claimed before the lock is released
    }
    lk.unlock();
    if (timed) NRG_CUDA_TRY(cudaEventRecord(ea, ctx->stream));
    int rc = NRG_OK;
    switch (v) {
        case 0: rc = launch_variant<kWM[0], kWN[0]>(ctx, 0, dp.as<GemmProblem>(), dq.as<int>(), np, live, prefix, dq); break;
        case 1: rc = launch_variant<kWM[1], kWN[1]>(ctx, 0, dp.as<GemmProblem>(), dq.as<int>(), np, live, prefix, dq); break;
        case 2: rc = launch_variant<kWM[2], kWN[2]>(ctx, 0, dp.as<GemmProblem>(), dq.as<int>(), np, live, prefix, dq); break;
        default: rc = launch_variant<kWM[3], kWN[3]>(ctx, 0, dp.as<GemmProblem>(), dq.as<int>(), np, live, prefix, dq); break;
    }
    if (timed) {
        const bool rec = rc == NRG_OK && cudaEventRecord(eb, ctx->stream) == cudaSuccess;
        lk.lock();
        if (rec) {
            tu.pending.push_back({key, v, ea, eb, gflop});
        } else {
            tu.table[key].inflight[v]--;
            tu.free_events.push_back(ea);
            tu.free_events.push_back(eb);
        }
    }
    return rc;
}

int GemmTuner::event(cudaEvent_t* e) {
    if (!free_events.empty()) {
        *e = free_events.back();
        free_events.pop_back();
        return NRG_OK;
    }
    NRG_CUDA_TRY(cudaEventCreate(e));
    return NRG_OK;
}

}  // namespace nrg
