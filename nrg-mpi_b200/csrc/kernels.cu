// Element kernels of the NRG hot path: sector Hamiltonian assembly, the post-eigensolver
// shift and chop, the sparse f^dagger gather, spike weights with log-grid binning, and
// small helpers.  All arithmetic is FP64.
#include "internal.hpp"

#include <math.h>

namespace nrg {
namespace {

constexpr int kMaxChain = 8;

struct AsmParams {
    int nb_old, nVar, nOps, nChain, nCM, flag_BCS, nsec, rec;
    double sqrtL;
    double cdiag[kMaxChain];   // chain_diagonal(iteration+1, c)
    double cnond[kMaxChain];   // chain_nondiagonal(iteration, c)
    double cbcs[kMaxChain];    // chain_BCS(iteration+1, c)
};

// Block Hamiltonian of diagonalization.F90:162-262.  One block per column of one sector.
// Products are rounded one at a time (no fused multiply-add) in the reference's order.
__global__ void k_assemble(const SyevSector* __restrict__ secs, const long long* __restrict__ colPrefix,
                           const int* __restrict__ secStart, const int* __restrict__ bi,
                           const double* __restrict__ Eold, const double* __restrict__ IMold,
                           const int* __restrict__ operation, const int* __restrict__ dflag,
                           const int* __restrict__ dtype, const int* __restrict__ dch,
                           const int* __restrict__ dswp, const double* __restrict__ dcoef,
                           const int* __restrict__ bflag, const int* __restrict__ bch,
                           double* __restrict__ V, AsmParams P, int* status) {
    const long long col = blockIdx.x;
    int lo = 0, hi = P.nsec - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (colPrefix[mid] <= col) lo = mid; else hi = mid - 1;
    }
    const int s = lo;
    const SyevSector sec = secs[s];
    const int d = sec.n;
    const int j = (int)(col - colPrefix[s]);
    const int row0 = secStart[s];
    const int R = P.rec;
    const size_t nbo = (size_t)P.nb_old;
    // An entry whose indices fall outside their tables, or whose value is NaN or Inf (from
    // the previous eigenvalues, invariant matrices or chain), is reported in the status
    // word and stored as 0: the eigensolver then runs on a finite matrix (its result is
    // discarded by the caller, which reads the status).  The reference passes such input
    // to dsyev unchecked.
    for (int i = threadIdx.x; i < d; i += blockDim.x) {
        double v = 0.0;
        int bad = 0;
        if (i == j) {
            const int* r = bi + (size_t)(row0 + i) * R;
            const int op = r[P.nVar + 2] - 1, ref = r[P.nVar] - 1;
            if (ref < 0 || ref >= P.nb_old || op < 0 || op >= P.nOps) {
                bad = NRG_DEV_BAD_INDEX;
            } else {
                v = __dmul_rn(Eold[ref], P.sqrtL);
                for (int c = 0; c < P.nChain; ++c)
                    v = __dadd_rn(v, __dmul_rn((double)operation[op + (size_t)(P.nVar + c) * P.nOps], P.cdiag[c]));
            }
        } else {
            const int p = i < j ? i : j, q = i < j ? j : i;
            const int* rp = bi + (size_t)(row0 + p) * R;
            const int* rq = bi + (size_t)(row0 + q) * R;
            const int a = rp[P.nVar + 2] - 1, b = rq[P.nVar + 2] - 1;
            const int refp = rp[P.nVar] - 1, refq = rq[P.nVar] - 1;
            if (a < 0 || a >= P.nOps || b < 0 || b >= P.nOps) {
                bad = NRG_DEV_BAD_INDEX;
            } else {
                const int idx = a * P.nOps + b;
                const bool sw = dswp[idx] != 0;
                const int ir = sw ? refq : refp, jr = sw ? refp : refq;
                if (dflag[idx]) {
                    const int t = dtype[idx] - 1, ch = dch[idx] - 1;
                    if (ir < 0 || jr < 0 || ir >= P.nb_old || jr >= P.nb_old || t < 0 || t >= P.nCM ||
                        ch < 0 || ch >= P.nChain)
                        bad = NRG_DEV_BAD_INDEX;
                    else
                        v = __dmul_rn(__dmul_rn(P.cnond[ch], dcoef[idx]),
                                      IMold[(size_t)jr + (size_t)ir * nbo + (size_t)t * nbo * nbo]);
                }
                if (!bad && P.flag_BCS && bflag[idx] && ir == jr) {
                    const int ch = bch[idx] - 1;
                    if (ch >= 0 && ch < P.nChain) v = P.cbcs[ch];
                }
            }
        }
        if (!bad && !isfinite(v)) bad = NRG_DEV_NONFINITE;
        if (bad) {
            atomicOr(status, bad);
            v = 0.0;
        }
        V[sec.a_off + (size_t)i + (size_t)j * d] = v;
    }
}

// minimum of E and the ground-state energy eigenvalue(1) before the shift
__global__ void k_min(const double* __restrict__ E, int n, double* out) {
    __shared__ double red[32];
    double m = INFINITY;
    for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmin(m, E[i]);
    for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = INFINITY;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r = fmin(r, red[w]);
        out[0] = r;
        out[1] = E[0];
    }
}

// diagonalization.F90:353-356
__global__ void k_shift(double* __restrict__ E, int n, const double* __restrict__ mn) {
    const double m = mn[0];
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double e = E[i] - m;
        if (e <= 1.0e-12) e = 0.0;
        E[i] = e;
    }
}

// diagonalization.F90:273-280
__global__ void k_chop(double* __restrict__ V, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        if (fabs(V[i]) < 1.0e-14) V[i] = 0.0;
    }
}

// T(i, j) = sum_b coef(a_i, b, t) V_R(rowOf(R, b, var_i), j), the sparse C_t of
// invariantMatrixDGEMM.F90:236-256 applied to V_R(:, 1:k_R)
__global__ void k_im_gather(const ImGatherProb* __restrict__ probs, const long long* __restrict__ prefix,
                            int nprob, const int* __restrict__ bi, int rec, int nVar, int nOps, int nCM,
                            const int* __restrict__ lst, const int* __restrict__ lstOff,
                            const int* __restrict__ imflag, const double* __restrict__ imcoef,
                            const double* __restrict__ V, double* __restrict__ T, long long total) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        int lo = 0, hi = nprob - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (prefix[mid] <= e) lo = mid; else hi = mid - 1;
        }
        const ImGatherProb pr = probs[lo];
        const long long loc = e - prefix[lo];
        const int i = (int)(loc % pr.dL), j = (int)(loc / pr.dL);
        const int* r = bi + (size_t)(pr.startL + i) * rec;
        const int a = r[nVar + 2] - 1, var = r[nVar + 1];
        double s = 0.0;
        for (int b = 0; b < nOps; ++b) {
            const int idx = (a * nOps + b) * nCM + pr.t;
            if (!imflag[idx]) continue;
            const int o0 = lstOff[pr.R * nOps + b], o1 = lstOff[pr.R * nOps + b + 1];
            if (var < 1 || var > o1 - o0) continue;
            const int row = lst[o0 + var - 1];
            s = fma(imcoef[idx], V[pr.vR_off + (size_t)row + (size_t)j * pr.dR], s);
        }
        T[pr.t_off + loc] = s;
    }
}

// spike weights w = S * Y (or S^2/pf at T=0) at energies sgn*(E_k - cE*E_l)*scale,
// binned like binningSpike (module.F90:1210-1254); raw sums per (matrix, sign).
// One block per tile of 32 k x 64 l spikes of one problem: the tile's bins are first
// accumulated in a shared-memory window (when they span at most kSpkWin bins), then
// added to the global bins once per touched bin; the raw sum takes one add per block.
constexpr int kSpkTK = 32, kSpkTL = 64, kSpkWin = 4096;

__global__ void __launch_bounds__(256) k_spikes(const SpikeProb* __restrict__ probs,
                                                const long long* __restrict__ tilePrefix, int nprob,
                                                const double* __restrict__ W, const double* __restrict__ E,
                                                int nbin, double* __restrict__ binPos, double* __restrict__ binNeg,
                                                double* __restrict__ tot, const double* __restrict__ Pw) {
    __shared__ double hist[kSpkWin];
    __shared__ double rs[8];
    __shared__ int rmin[8], rmax[8];
    const long long bid = blockIdx.x;
    int lo = 0, hi = nprob - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (tilePrefix[mid] <= bid) lo = mid; else hi = mid - 1;
    }
    const SpikeProb pr = probs[lo];
    const long long tix = bid - tilePrefix[lo];
    const int ntk = (pr.kk + kSpkTK - 1) / kSpkTK;
    const int tk = (int)(tix % ntk), tl = (int)(tix / ntk);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int k1 = tk * kSpkTK + lane;
    const int lb = tl * kSpkTL + warp;
    const double ek = k1 < pr.kk ? E[pr.ek_off + k1] : 0.0;
    int ia[8], ib[8];
    double wa[8], wv[8];
    double wsum = 0.0;
    int bmin = 0x7fffffff, bmax = -1;
#pragma unroll
    for (int u = 0; u < 8; ++u) {
        const int l = lb + 8 * u;
        ia[u] = -1;
        ib[u] = -1;
        wa[u] = 0.0;
        wv[u] = 0.0;
        if (k1 < pr.kk && l < pr.nl) {
            const long long loc = (long long)k1 + (long long)l * pr.kk;
            const double sv = W[pr.s_off + loc];
            const double el = E[pr.el_off + (long long)l * pr.lstride];
            const double en = pr.sgn * ((ek - pr.cE * el) * pr.scale);
            double w;
            if (!pr.fdm) {
                w = (pr.y_off >= 0) ? sv * W[pr.y_off + loc] : sv * sv * pr.invpf;
            } else {
                // both terms of a pair sit at omega = en: the term of the state that gains
                // the particle (x) enters the positive bins for omega >= 0, the term of the
                // state that loses it (y) for omega > 0; the rest goes to the negative bins
                const bool inx = pr.toPos ? (en >= 0.0) : (en < 0.0);
                const bool iny = pr.toPos ? (en > 0.0) : (en <= 0.0);
                const double pk = Pw[pr.ek_off + k1], pl = Pw[pr.el_off + (long long)l * pr.lstride];
                const double px = pr.k_is_y ? pl : pk, py = pr.k_is_y ? pk : pl;
                w = sv * sv * ((inx ? px : 0.0) + (iny ? py : 0.0));
                if (pr.y_off >= 0 && (pr.k_is_y ? iny : inx)) w += sv * W[pr.y_off + loc];
            }
            wsum += w;
            // binningSpike
            const double position = (log10(fabs(en)) - (-15.0)) * 1000.0 + 1.0;
            long long pref = (long long)position;   // int(): truncation toward zero
            int i1 = 0;
            if (position <= 0.0) i1 = 1;
            else if (position >= (double)nbin) i1 = nbin;
            if (pref <= 0) pref = 1;
            if (i1 > 0) {
                ia[u] = i1;
                wa[u] = w;
            } else {
                const double wb = position - (double)pref;
                ia[u] = (int)pref;
                wa[u] = w * (1.0 - wb);
                ib[u] = (int)pref + 1;
                wv[u] = w * wb;
            }
            bmin = min(bmin, ia[u]);
            bmax = max(bmax, ib[u] >= 0 ? ib[u] : ia[u]);
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        wsum += __shfl_xor_sync(0xffffffffu, wsum, o);
        bmin = min(bmin, __shfl_xor_sync(0xffffffffu, bmin, o));
        bmax = max(bmax, __shfl_xor_sync(0xffffffffu, bmax, o));
    }
    if (lane == 0) { rs[warp] = wsum; rmin[warp] = bmin; rmax[warp] = bmax; }
    __syncthreads();
    double ws = 0.0;
    int wmin = 0x7fffffff, wmax = -1;
    for (int q = 0; q < 8; ++q) { ws += rs[q]; wmin = min(wmin, rmin[q]); wmax = max(wmax, rmax[q]); }
    if (tid == 0 && wmax >= 0) atomicAdd(&tot[2 * pr.m + (pr.toPos ? 1 : 0)], ws);
    if (wmax < 0) return;
    double* cont = (pr.toPos ? binPos : binNeg) + ((size_t)pr.m * nbin - 1);
    const int win = wmax - wmin + 1;
    if (win <= kSpkWin) {
        for (int i = tid; i < win; i += 256) hist[i] = 0.0;
        __syncthreads();
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            if (ia[u] >= 0) atomicAdd(&hist[ia[u] - wmin], wa[u]);
            if (ib[u] >= 0) atomicAdd(&hist[ib[u] - wmin], wv[u]);
        }
        __syncthreads();
        for (int i = tid; i < win; i += 256)
            if (hist[i] != 0.0) atomicAdd(&cont[wmin + i], hist[i]);
    } else {
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            if (ia[u] >= 0) atomicAdd(&cont[ia[u]], wa[u]);
            if (ib[u] >= 0) atomicAdd(&cont[ib[u]], wv[u]);
        }
    }
}

// calcThermo (module.F90:1931-1982) on one iteration's eigenvalues in sector order, before
// truncation (postprocess.F90:62): Z, E = sum bE e^-bE, <Sz^2>, <Sz> with bE = betabar E,
// then C = sum (bE - E/Z)^2 e^-bE / Z (the fluctuation form), S = E/Z + ln Z and
// X = <Sz^2> - <Sz>^2.  One block; partial sums per thread, combined in a fixed order.
// tab: sector start | dimension | 2 Sz, nsub entries each.
__device__ __forceinline__ void thermo_sum(double* v, int nv, double (*red)[32]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int q = 0; q < nv; ++q)
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
    __syncthreads();
    if (lane == 0)
        for (int q = 0; q < nv; ++q) red[q][warp] = v[q];
    __syncthreads();
    for (int q = 0; q < nv; ++q) {
        double s = 0.0;
        for (int w = 0; w < nw; ++w) s += red[q][w];
        v[q] = s;
    }
}
__global__ void __launch_bounds__(512) k_thermo(const double* __restrict__ E, const int* __restrict__ tab,
                                                int nsub, double betabar, double* __restrict__ out) {
    __shared__ double red[4][32];
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    for (int s = 0; s < nsub; ++s) {
        const int s0 = tab[s], d = tab[nsub + s];
        const double sz = 0.5 * tab[2 * nsub + s];
        for (int i = threadIdx.x; i < d; i += blockDim.x) {
            const double bE = betabar * E[s0 + i];
            const double ex = exp(-bE);
            v[0] += ex;
            v[1] += bE * ex;
            v[2] += ex * sz * sz;
            v[3] += ex * sz;
        }
    }
    thermo_sum(v, 4, red);
    const double Z = v[0], em = v[1] / Z;
    double c[1] = {0.0};
    for (int s = 0; s < nsub; ++s) {
        const int s0 = tab[s], d = tab[nsub + s];
        for (int i = threadIdx.x; i < d; i += blockDim.x) {
            const double bE = betabar * E[s0 + i];
            c[0] += (bE - em) * (bE - em) * exp(-bE);
        }
    }
    thermo_sum(c, 1, red);
    if (threadIdx.x == 0) {
        out[0] = c[0] / Z;
        out[1] = em + log(Z);
        out[2] = v[2] / Z - (v[3] / Z) * (v[3] / Z);
    }
}

// log-Gaussian broadening of binned spikes (Bulla, Costi and Pruschke, Rev. Mod. Phys. 80,
// 395 (2008), Sec. V.A): A(w) = sum_i w_i P(w, E_i) with
// P(w, E) = exp(-b^2/4) / (b |E| sqrt(pi)) exp(-(ln(w/E)/b)^2) for w E > 0, else 0.
// bins: Fortran (nbin*nMat, 2) (energies, then weights; column stride ld); one block per
// (output frequency, matrix type), threads over the bins, partial sums in a fixed order.
__global__ void __launch_bounds__(256) k_broaden(const double* __restrict__ bins, int nbin, long long ld,
                                                 double b, const double* __restrict__ omega, int nw,
                                                 double* __restrict__ A) {
    __shared__ double red[8];
    const int k = blockIdx.x % nw, m = blockIdx.x / nw;
    const double w = omega[k];
    const double* E = bins + (size_t)m * nbin;
    const double* W = bins + ld + (size_t)m * nbin;
    double s = 0.0;
    for (int i = threadIdx.x; i < nbin; i += blockDim.x) {
        const double wi = W[i], ei = E[i];
        if (wi == 0.0 || !(w * ei > 0.0)) continue;
        const double x = log(w / ei) / b;
        s += wi * exp(-x * x) / fabs(ei);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t += red[q];
        A[(size_t)m * nw + k] = t * exp(-0.25 * b * b) / (b * sqrt(3.14159265358979323846));
    }
}

// element e of the concatenated runs: segment by binary search over the element prefix,
// then run and offset; consecutive threads read consecutive doubles of a run
__global__ void k_gather_segs(const double* __restrict__ src, double* __restrict__ dst, long long ld,
                              const HostSeg* __restrict__ segs, const long long* __restrict__ prefix, int nseg,
                              long long total, int packed) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        int lo = 0, hi = nseg - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (prefix[mid] <= e) lo = mid; else hi = mid - 1;
        }
        const HostSeg g = segs[lo];
        const long long loc = e - prefix[lo];
        const long long p = g.off + (loc / g.len) * ld + loc % g.len;
        dst[p] = src[packed ? e : p];
    }
}

__global__ void k_scaled_gather(const ScaledGather* __restrict__ jobs, const long long* __restrict__ prefix, int nj,
                                long long total, double* __restrict__ dst, const double* __restrict__ V,
                                const int* __restrict__ rows, const double* __restrict__ P) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        int lo = 0, hi = nj - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (prefix[mid] <= e) lo = mid; else hi = mid - 1;
        }
        const ScaledGather g = jobs[lo];
        const long long loc = e - prefix[lo];
        const int i = (int)(loc % g.n), j = (int)(loc / g.n);
        const int r = rows[g.rows + i];
        dst[g.dst + loc] = V[g.v + (long long)r + (long long)(g.c0 + j) * g.ld] * P[g.p + j];
    }
}

__global__ void k_fill(double* p, long long n, double v) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) p[i] = v;
}
__global__ void k_add(double* dst, const double* src, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) dst[i] += src[i];
}
// per matrix type: sum of the bins (sequential per type, deterministic)
__global__ void k_sum_bins(const double* bins, int nbin, double* out) {
    __shared__ double red[32];
    const int m = blockIdx.x;
    double s = 0.0;
    for (int i = threadIdx.x; i < nbin; i += blockDim.x) s += bins[(size_t)m * nbin + i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r += red[w];
        out[m] = r;
    }
}
// sum of the diagonals of row-major square blocks
__global__ void k_trace(const double* rdm, const long long* offs, const int* dims, int nblk, double* out) {
    __shared__ double red[32];
    double s = 0.0;
    for (int b = 0; b < nblk; ++b) {
        const int n = dims[b];
        for (int i = threadIdx.x; i < n; i += blockDim.x) s += rdm[offs[b] + (long long)i * n + i];
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r += red[w];
        out[0] = r;
    }
}
__global__ void k_gather_rows(double* dst, long long dst_ld, const double* src, long long src_ld,
                              const int* rows, int nrows, int ncols) {
    const long long total = (long long)nrows * ncols;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(e % nrows), j = (int)(e / nrows);
        dst[(size_t)i + (size_t)j * dst_ld] = src[(size_t)rows[i] + (size_t)j * src_ld];
    }
}

int grid_for(long long n, int threads) {
    long long g = (n + threads - 1) / threads;
    if (g < 1) g = 1;
    if (g > 148 * 32) g = 148 * 32;
    return (int)g;
}

}  // namespace

int run_assemble(nrg_context* ctx, int iteration, const Sectors& S, const SyevSector* d_secs,
                 const long long* d_colPrefix, const int* d_secStart, int nsec, long long ncols,
                 const double* d_Eold, int nb_old, const double* d_IMold, double* d_V) {
    const Model& M = ctx->model;
    if (M.nChain > kMaxChain) return NRG_ERR_UNSUPPORTED;
    AsmParams P;
    P.nb_old = nb_old; P.nVar = M.nVar; P.nOps = M.nOps; P.nChain = M.nChain; P.nCM = M.nCM;
    P.flag_BCS = M.flag_BCS; P.nsec = nsec; P.rec = M.nVar + 3;
    P.sqrtL = sqrt(M.Lambda);
    for (int c = 0; c < kMaxChain; ++c) {
        P.cdiag[c] = c < M.nChain ? M.cd(iteration + 1, c) : 0.0;
        P.cnond[c] = c < M.nChain ? M.cn(iteration, c) : 0.0;
        P.cbcs[c] = (c < M.nChain && M.flag_BCS) ? M.cbcs(iteration + 1, c) : 0.0;
    }
    if (ncols == 0) return NRG_OK;
    k_assemble<<<(unsigned)ncols, 128, 0, ctx->stream>>>(
        d_secs, d_colPrefix, d_secStart, S.d_bi.as<int>(),
        d_Eold, d_IMold, M.d_operation.as<int>(), M.d_dflag.as<int>(), M.d_dtype.as<int>(),
        M.d_dch.as<int>(), M.d_dswp.as<int>(), M.d_dcoef.as<double>(), M.d_bflag.as<int>(),
        M.d_bch.as<int>(), d_V, P, ctx->d_status.as<int>());
    ctx->launches++;
    NRG_CUDA_TRY(cudaGetLastError());
    return NRG_OK;
}

int run_eig_shift(nrg_context* ctx, double* d_E, int nb, double* d_min_and_gs) {
    k_min<<<1, 1024, 0, ctx->stream>>>(d_E, nb, d_min_and_gs);
    k_shift<<<grid_for(nb, 256), 256, 0, ctx->stream>>>(d_E, nb, d_min_and_gs);
    ctx->launches += 2;
    NRG_CUDA_TRY(cudaGetLastError());
    return NRG_OK;
}

int run_eig_chop(nrg_context* ctx, long long sizeV, double* d_V, cudaStream_t st) {
    if (sizeV <= 0) return NRG_OK;
    k_chop<<<grid_for(sizeV, 256), 256, 0, st ? st : ctx->stream>>>(d_V, sizeV);
    ctx->launches++;
    NRG_CUDA_TRY(cudaGetLastError());
    return NRG_OK;
}

int run_im_gather(nrg_context* ctx, const Sectors& S, std::vector<ImGatherProb>& probs,
                  const double* d_V, double* d_T) {
    const Model& M = ctx->model;
    const int np = (int)probs.size();
    if (np == 0) return NRG_OK;
    std::vector<long long> prefix(np);
    long long total = 0;
    for (int p = 0; p < np; ++p) { prefix[p] = total; total += (long long)probs[p].dL * probs[p].kR; }
    if (total == 0) return NRG_OK;
    DevBuf& dp = ctx->scratch.b[16];
    DevBuf& dq = ctx->scratch.b[17];
    NRG_TRY(dp.ensure(sizeof(ImGatherProb) * np));
    NRG_TRY(dq.ensure(sizeof(long long) * np));
    NRG_TRY(h2d_async(ctx, dp.p, probs.data(), sizeof(ImGatherProb) * np));
    NRG_TRY(h2d_async(ctx, dq.p, prefix.data(), sizeof(long long) * np));
    k_im_gather<<<grid_for(total, 256), 256, 0, ctx->stream>>>(
        dp.as<ImGatherProb>(), dq.as<long long>(), np, S.d_bi.as<int>(), M.nVar + 3, M.nVar, M.nOps,
        M.nCM, S.d_lst.as<int>(), S.d_lstOff.as<int>(), M.d_imflag.as<int>(), M.d_imcoef.as<double>(),
        d_V, d_T, total);
    ctx->launches++;
    NRG_CUDA_TRY(cudaGetLastError());
    return NRG_OK;
}

int run_spikes(nrg_context* ctx, std::vector<SpikeProb>& probs, const double* d_work,
               const double* d_E, int nbin, int nMat, double* d_binPos, double* d_binNeg,
               double* d_tot, const double* d_P) {
    (void)nMat;
    const int np = (int)probs.size();
    if (np == 0) return NRG_OK;
    std::vector<long long> prefix(np);
    long long total = 0;
    for (int p = 0; p < np; ++p) {
        prefix[p] = total;
        total += (long long)((probs[p].kk + kSpkTK - 1) / kSpkTK) * ((probs[p].nl + kSpkTL - 1) / kSpkTL);
    }
    if (total == 0) return NRG_OK;
    if (total > 0x7fffffffLL) return NRG_ERR_TOO_LARGE;
    DevBuf& dp = ctx->scratch.b[18];
    DevBuf& dq = ctx->scratch.b[19];
    NRG_TRY(dp.ensure(sizeof(SpikeProb) * np));
    NRG_TRY(dq.ensure(sizeof(long long) * np));
    NRG_TRY(h2d_async(ctx, dp.p, probs.data(), sizeof(SpikeProb) * np));
    NRG_TRY(h2d_async(ctx, dq.p, prefix.data(), sizeof(long long) * np));
    for (const auto& p : probs)
        if (p.fdm && !d_P) {
            nrg_set_error_message("full-density-matrix spikes without weights");
            return NRG_ERR_INVALID;
        }
    k_spikes<<<(unsigned)total, 256, 0, ctx->stream>>>(dp.as<SpikeProb>(), dq.as<long long>(), np, d_work, d_E, nbin,
                                                     d_binPos, d_binNeg, d_tot, d_P);
    ctx->launches++;
    NRG_CUDA_TRY(cudaGetLastError());
    return NRG_OK;
}

int run_thermo(nrg_context* ctx, const Sectors& S, const double* d_E, double* d_out) {
    const Model& M = ctx->model;
    const int nsub = S.nsub, nVar = S.nVar;
    std::vector<int> tab(3 * (size_t)nsub);
    for (int s = 0; s < nsub; ++s) {
        int sz = 0;
        for (int v = M.cb[1]; v <= M.cb[3]; ++v) sz += S.qn[(size_t)s * nVar + v - 1];
        tab[s] = S.start[s];
        tab[nsub + s] = S.dim[s];
        tab[2 * nsub + s] = sz;
    }
    DevBuf& b = ctx->scratch.b[38];
    NRG_TRY(b.ensure(sizeof(int) * tab.size()));
    NRG_TRY(h2d_async(ctx, b.p, tab.data(), sizeof(int) * tab.size()));
    k_thermo<<<1, 512, 0, ctx->stream>>>(d_E, b.as<int>(), nsub, kBetabar, d_out);
    ctx->launches++;
    NRG_CUDA_TRY(cudaGetLastError());
    return NRG_OK;
}

int run_broaden(nrg_context* ctx, const double* d_bins, int nbin, int nMat, double b, const double* d_omega,
                int nw, double* d_A) {
    if (nw <= 0 || nMat <= 0) return NRG_OK;
    const long long blocks = (long long)nw * nMat;
    if (blocks > 0x7fffffffLL) return NRG_ERR_TOO_LARGE;
    k_broaden<<<(unsigned)blocks, 256, 0, ctx->stream>>>(d_bins, nbin, (long long)nbin * nMat, b, d_omega, nw, d_A);
    ctx->launches++;
    NRG_CUDA_TRY(cudaGetLastError());
    return NRG_OK;
}

int run_gather_segs(nrg_context* ctx, const double* src, double* dst, long long ld,
                    const std::vector<HostSeg>& segs, long long* bytes, bool packed) {
    const int ns = (int)segs.size();
    *bytes = 0;
    if (ns == 0) return NRG_OK;
    std::vector<long long> prefix(ns);
    long long total = 0;
    for (int i = 0; i < ns; ++i) {
        prefix[i] = total;
        total += (long long)segs[i].len * segs[i].count;
    }
    if (total == 0) return NRG_OK;
    DevBuf& bs = ctx->scratch.b[20];
    DevBuf& bp = ctx->scratch.b[23];
    NRG_TRY(bs.ensure(sizeof(HostSeg) * ns));
    NRG_TRY(bp.ensure(sizeof(long long) * ns));
    NRG_TRY(h2d_async(ctx, bs.p, segs.data(), sizeof(HostSeg) * ns));
    NRG_TRY(h2d_async(ctx, bp.p, prefix.data(), sizeof(long long) * ns));
    const long long grid = std::min<long long>((total + 255) / 256, 148LL * 16);
    k_gather_segs<<<(unsigned)grid, 256, 0, ctx->stream>>>(src, dst, ld, bs.as<HostSeg>(), bp.as<long long>(), ns,
                                                          total, packed ? 1 : 0);
    ctx->launches++;
    NRG_CUDA_TRY(cudaGetLastError());
    *bytes = total * (long long)sizeof(double);
    return NRG_OK;
}

int run_scaled_gather(nrg_context* ctx, const std::vector<ScaledGather>& jobs, double* dst, const double* V,
                      const int* rows, const double* P) {
    const int nj = (int)jobs.size();
    if (nj == 0) return NRG_OK;
    std::vector<long long> prefix(nj);
    long long total = 0;
    for (int i = 0; i < nj; ++i) {
        prefix[i] = total;
        total += (long long)jobs[i].n * jobs[i].nc;
    }
    if (total == 0) return NRG_OK;
    DevBuf& bj = ctx->scratch.b[40];
    DevBuf& bp = ctx->scratch.b[41];
    NRG_TRY(bj.ensure(sizeof(ScaledGather) * nj));
    NRG_TRY(bp.ensure(sizeof(long long) * nj));
    NRG_TRY(h2d_async(ctx, bj.p, jobs.data(), sizeof(ScaledGather) * nj));
    NRG_TRY(h2d_async(ctx, bp.p, prefix.data(), sizeof(long long) * nj));
    const long long grid = std::min<long long>((total + 255) / 256, 148LL * 16);
    k_scaled_gather<<<(unsigned)grid, 256, 0, ctx->stream>>>(bj.as<ScaledGather>(), bp.as<long long>(), nj, total, dst,
                                                            V, rows, P);
    ctx->launches++;
    NRG_CUDA_TRY(cudaGetLastError());
    return NRG_OK;
}

int run_fill(nrg_context* ctx, double* p, long long n, double v) {
    if (n <= 0) return NRG_OK;
    k_fill<<<grid_for(n, 256), 256, 0, ctx->stream>>>(p, n, v);
    ctx->launches++;
    NRG_CUDA_TRY(cudaGetLastError());
    return NRG_OK;
}
int run_add(nrg_context* ctx, double* dst, const double* src, long long n) {
    if (n <= 0) return NRG_OK;
    k_add<<<grid_for(n, 256), 256, 0, ctx->stream>>>(dst, src, n);
    ctx->launches++;
    NRG_CUDA_TRY(cudaGetLastError());
    return NRG_OK;
}
int run_sum_bins(nrg_context* ctx, const double* bins, int nbin, int nMat, double* out) {
    if (nMat <= 0) return NRG_OK;
    k_sum_bins<<<nMat, 1024, 0, ctx->stream>>>(bins, nbin, out);
    ctx->launches++;
    NRG_CUDA_TRY(cudaGetLastError());
    return NRG_OK;
}
int run_trace(nrg_context* ctx, const double* rdm, const long long* d_offs, const int* d_dims,
              int nblk, double* out) {
    k_trace<<<1, 1024, 0, ctx->stream>>>(rdm, d_offs, d_dims, nblk, out);
    ctx->launches++;
    NRG_CUDA_TRY(cudaGetLastError());
    return NRG_OK;
}
int run_gather_rows(nrg_context* ctx, double* dst, long long dst_ld, const double* src,
                    long long src_ld, const int* d_rows, int nrows, int ncols) {
    const long long n = (long long)nrows * ncols;
    if (n <= 0) return NRG_OK;
    k_gather_rows<<<grid_for(n, 256), 256, 0, ctx->stream>>>(dst, dst_ld, src, src_ld, d_rows, nrows, ncols);
    ctx->launches++;
    NRG_CUDA_TRY(cudaGetLastError());
    return NRG_OK;
}

}  // namespace nrg
