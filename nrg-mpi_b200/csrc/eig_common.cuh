// Device building blocks of the FP64 symmetric eigensolver shared by the one-block-per-
// sector kernel (eig.cu) and the multi-kernel pipeline for large sectors (eig_large.cu):
// reductions, the divide-and-conquer merge in phases, and the secular-equation solver.
#pragma once
#include "common.cuh"
#include "cta_gemm.cuh"

#include <math.h>
#include <type_traits>

namespace {

constexpr double kEps = 1.1102230246251565e-16;

// a whole block or one warp
struct BlockG {
    __device__ int rank() const { return threadIdx.x; }
    __device__ int size() const { return blockDim.x; }
    __device__ void sync() const { __syncthreads(); }
};
struct WarpG {
    int lane;
    __device__ int rank() const { return lane; }
    __device__ int size() const { return 32; }
    __device__ void sync() const { __syncwarp(); }
};

__device__ double block_sum(double v, double* red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
    const int nw = blockDim.x >> 5;
    for (int i = 0; i < nw; ++i) s += red[i];   // same order in every thread
    return s;
}
__device__ double block_max(double v, double* red) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
    const int nw = blockDim.x >> 5;
    for (int i = 0; i < nw; ++i) s = fmax(s, red[i]);
    return s;
}
__device__ double group_max(BlockG, double v, double* red) { return block_max(v, red); }
__device__ double group_max(WarpG, double v, double*) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// scratch arrays of one sector, each of length n, indexed by absolute row
struct Scratch {
    double *z, *ds, *zs, *dd, *zz, *tau, *zh, *vals, *rc, *rs;
    int *perm, *nd, *df, *org, *pos, *ra, *rb, *mk, *mr, *mf;
};

__device__ Scratch scratch_at(double* vec, int* I, int n) {
    // vec: D, E, TAU, then the merge arrays; I: the integer arrays
    Scratch S;
    S.z = vec + 3 * n; S.ds = vec + 4 * n; S.zs = vec + 5 * n; S.dd = vec + 6 * n;
    S.zz = vec + 7 * n; S.tau = vec + 8 * n; S.zh = vec + 9 * n; S.vals = vec + 10 * n;
    S.rc = vec + 11 * n; S.rs = vec + 12 * n;
    S.perm = I; S.nd = I + n; S.df = I + 2 * n; S.org = I + 3 * n; S.pos = I + 4 * n;
    S.ra = I + 5 * n; S.rb = I + 6 * n; S.mk = I + 7 * n; S.mr = I + 8 * n; S.mf = I + 9 * n;
    return S;
}

// The same vectors for a range of at most cap rows in shared memory, indexed from the
// start of the range: cap doubles for D, then 10 cap doubles and 10 cap ints (16 cap
// doubles in all, from dsm).  The merges' serial and iterative parts (deflation scan,
// secular roots, ranks) then wait on shared memory instead of L2.
constexpr int kDcSmemDoubles = 16;
__device__ Scratch scratch_smem(double* dsm, int cap) {
    Scratch S;
    double* v = dsm + cap;
    int* I = reinterpret_cast<int*>(dsm + 11 * cap);
    S.z = v; S.ds = v + cap; S.zs = v + 2 * cap; S.dd = v + 3 * cap; S.zz = v + 4 * cap;
    S.tau = v + 5 * cap; S.zh = v + 6 * cap; S.vals = v + 7 * cap; S.rc = v + 8 * cap; S.rs = v + 9 * cap;
    S.perm = I; S.nd = I + cap; S.df = I + 2 * cap; S.org = I + 3 * cap; S.pos = I + 4 * cap;
    S.ra = I + 5 * cap; S.rb = I + 6 * cap; S.mk = I + 7 * cap; S.mr = I + 8 * cap; S.mf = I + 9 * cap;
    return S;
}

// How the O(K) sums of one secular root, one zhat entry or one rank-one eigenvector are
// split: one thread runs the whole sum, or the 32 lanes of a warp take every 32nd term
// and combine them with a butterfly (every lane ends with the same value).
struct SeqLanes {
    __device__ int first() const { return 0; }
    __device__ int step() const { return 1; }
    __device__ bool leader() const { return true; }
    __device__ double sum(double v) const { return v; }
    __device__ double prod(double v) const { return v; }
};
// G aligned lanes of a warp (G = 2, 4, ..., 32) share one item; the shuffles name only
// the group's lanes, so groups of one warp may leave their loops at different times
template <int G>
struct GroupLanes {
    int lane;   // lane index in the warp
    __device__ int first() const { return lane & (G - 1); }
    __device__ int step() const { return G; }
    __device__ bool leader() const { return (lane & (G - 1)) == 0; }
    __device__ unsigned mask() const {
        return G == 32 ? 0xffffffffu : (((1u << G) - 1u) << (lane & ~(G - 1)));
    }
    __device__ double sum(double v) const {
        for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask(), v, o);
        return v;
    }
    __device__ double prod(double v) const {
        for (int o = G / 2; o > 0; o >>= 1) v *= __shfl_xor_sync(mask(), v, o);
        return v;
    }
};
using WarpLanes = GroupLanes<32>;
// lanes per item inside the one-block merges
constexpr int kMergeLanes = 4;

// Root j of 1 + rho * sum_i zz_i^2 / (dd_i - lambda) = 0 (rho > 0, dd ascending, zz != 0),
// returned as lambda = dd[org] + tau with org the pole nearer to the root, so that every
// difference dd_i - lambda = (dd_i - dd[org]) - tau keeps full relative accuracy.
// Iteration: the two-pole rational model of the secular function (the poles bounding
// the root carry the near terms, Bunch-Nielsen-Sorensen), solved as a quadratic, kept
// inside a bisection bracket; at most 100 steps.
template <class R>
__device__ void secular_root(R r, int K, const double* dd, const double* zz, double rho, int j,
                             int* org, double* tau, int* status) {
    double zsq = 0.0;
    for (int i = r.first(); i < K; i += r.step()) zsq += zz[i] * zz[i];
    zsq = r.sum(zsq);
    int o;
    double lo, hi;
    auto gval = [&](int oo, double t) {
        double s = 0.0;
        const double base = dd[oo];
        for (int i = r.first(); i < K; i += r.step()) s += zz[i] * zz[i] / ((dd[i] - base) - t);
        return 1.0 + rho * r.sum(s);
    };
    if (j < K - 1) {
        const double gap = dd[j + 1] - dd[j];
        if (gval(j, 0.5 * gap) >= 0.0) { o = j; lo = 0.0; hi = 0.5 * gap; }
        else { o = j + 1; lo = -0.5 * gap; hi = 0.0; }
    } else {
        o = K - 1;
        const double up = rho * zsq;
        if (gval(o, 0.5 * up) >= 0.0) { lo = 0.0; hi = 0.5 * up; } else { lo = 0.5 * up; hi = up; }
    }
    const double base = dd[o];
    double t = 0.5 * (lo + hi);
    for (int it = 0; it < 100; ++it) {
        double psi = 0.0, dpsi = 0.0, phi = 0.0, dphi = 0.0;
        for (int i = r.first(); i < K; i += r.step()) {
            const double rdel = 1.0 / ((dd[i] - base) - t);
            const double q = zz[i] * zz[i] * rdel;
            if (i <= j) { psi += q; dpsi += q * rdel; } else { phi += q; dphi += q * rdel; }
        }
        psi = r.sum(psi); dpsi = r.sum(dpsi); phi = r.sum(phi); dphi = r.sum(dphi);
        psi *= rho; dpsi *= rho; phi *= rho; dphi *= rho;
        const double f = 1.0 + psi + phi;
        if (f > 0.0) hi = t;
        else if (f < 0.0) lo = t;
        else break;
        if (fabs(f) <= 8.0 * K * kEps * (1.0 + fabs(psi) + fabs(phi))) break;
        const double D1 = (dd[j] - base) - t;
        bool ok = false;
        double eta = 0.0;
        if (j < K - 1) {
            const double D2 = (dd[j + 1] - base) - t;
            const double b = dpsi * D1 * D1, a = psi - b / D1;
            const double e2 = dphi * D2 * D2, c = phi - e2 / D2;
            const double C = 1.0 + a + c;
            const double A2 = C, B2 = -(C * (D1 + D2) + b + e2), C2 = D1 * D2 * f;
            const double disc = B2 * B2 - 4.0 * A2 * C2;
            if (disc >= 0.0 && A2 != 0.0) {
                const double sq = sqrt(disc);
                const double qq = -0.5 * (B2 + (B2 >= 0.0 ? sq : -sq));
                const double r1 = qq / A2, r2 = (qq != 0.0) ? C2 / qq : r1;
                double best = 1e300;
                if (t + r1 > lo && t + r1 < hi) { best = r1; ok = true; }
                if (t + r2 > lo && t + r2 < hi && fabs(r2) < fabs(best)) { best = r2; ok = true; }
                eta = best;
            }
        } else {
            const double b = dpsi * D1 * D1, a = psi - b / D1;
            const double C = 1.0 + a;
            if (C > 0.0) {
                eta = ((dd[j] - base) + b / C) - t;
                ok = (t + eta > lo && t + eta < hi);
            }
        }
        const double tn = ok ? t + eta : 0.5 * (lo + hi);
        if (tn == t) break;
        t = tn;
        if (hi - lo <= 2.0 * kEps * fmax(fabs(lo), fabs(hi))) break;
    }
    if (r.leader()) {
        if (!(t == t)) atomicOr(status, NRG_DEV_SECULAR);
        *org = o;
        *tau = t;
    }
}

// dd_i - lambda_j
__device__ __forceinline__ double sec_delta(const double* dd, const int* org, const double* tau,
                                            int i, int j) {
    return (dd[i] - dd[org[j]]) - tau[j];
}

// ------------------------------------------------------------------------------------
// one divide-and-conquer merge of rows/cols [a, mid) and [mid, b) of Z (leading dim n),
// split into phases; (t, T) is the calling thread's rank among T threads on this merge
// ------------------------------------------------------------------------------------

// z vector, merge order, deflation (dlaed2-style), rotations, and the kept poles
template <class G>
__device__ void merge_prep(G g, int a, int mid, int b, int n, double* Z, const double* D,
                           const double* E, Scratch S, double* red) {
    const int t = g.rank(), T = g.size();
    const int nn = b - a, n1 = mid - a;
    const double beta = E[mid - 1];
    const double rho = 2.0 * fabs(beta);
    const double sg = beta >= 0.0 ? 1.0 : -1.0;
    const double r2 = 0.70710678118654752440;
    // z = [last row of Q1, sign(beta) * first row of Q2] / sqrt(2)
    for (int i = t; i < nn; i += T) {
        const int col = a + i;
        S.z[a + i] = (i < n1 ? Z[(size_t)(mid - 1) + (size_t)col * n]
                             : sg * Z[(size_t)mid + (size_t)col * n]) * r2;
    }
    // stable merge order of the two ascending halves (first half wins ties)
    for (int i = t; i < nn; i += T) {
        int rank;
        const double v = D[a + i];
        if (i < n1) {
            int lo = 0, hi = nn - n1;
            while (lo < hi) { const int m = (lo + hi) >> 1; if (D[mid + m] < v) lo = m + 1; else hi = m; }
            rank = i + lo;
        } else {
            int lo = 0, hi = n1;
            while (lo < hi) { const int m = (lo + hi) >> 1; if (D[a + m] <= v) lo = m + 1; else hi = m; }
            rank = (i - n1) + lo;
        }
        S.perm[a + rank] = i;
    }
    g.sync();
    double dm = 0.0, zm = 0.0;
    for (int r = t; r < nn; r += T) {
        const int p = S.perm[a + r];
        const double dv = D[a + p], zv = S.z[a + p];
        S.ds[a + r] = dv;
        S.zs[a + r] = zv;
        dm = fmax(dm, fabs(dv));
        zm = fmax(zm, fabs(zv));
    }
    dm = group_max(g, dm, red);
    zm = group_max(g, zm, red);
    const double tol = 8.0 * kEps * fmax(dm, zm);
    g.sync();
    if (t == 0) {
        int K = 0, ndf = 0, nrot = 0, jlam = -1;
        double* ds = S.ds + a;
        double* zs = S.zs + a;
        double zl = 0.0, dl = 0.0;   // z and d of the pending entry jlam
        for (int j = 0; j < nn; ++j) {
            const double zj = zs[j], dj = ds[j];
            if (rho * fabs(zj) <= tol) { S.df[a + ndf++] = j; continue; }
            if (jlam < 0) { jlam = j; zl = zj; dl = dj; continue; }
            // close poles: |(d_j - d_l) c s| <= tol with c = z_j / tau, s = -z_l / tau,
            // tau^2 = z_j^2 + z_l^2, tested without the square root and the divisions
            // (the rotation itself is rare)
            const double tt = dj - dl;
            if (fabs(tt) * fabs(zj * zl) <= tol * fma(zj, zj, zl * zl)) {
                const double tau = hypot(zj, zl);
                const double c_ = zj / tau, s_ = -zl / tau;
                zs[j] = tau;
                zs[jlam] = 0.0;
                S.ra[a + nrot] = S.perm[a + jlam];
                S.rb[a + nrot] = S.perm[a + j];
                S.rc[a + nrot] = c_;
                S.rs[a + nrot] = s_;
                ++nrot;
                const double tn = dl * c_ * c_ + dj * s_ * s_;
                const double dn = dl * s_ * s_ + dj * c_ * c_;
                ds[j] = dn;
                ds[jlam] = tn;
                S.df[a + ndf++] = jlam;
                jlam = j;
                zl = tau;
                dl = dn;
            } else {
                S.nd[a + K++] = jlam;
                jlam = j;
                zl = zj;
                dl = dj;
            }
        }
        if (jlam >= 0) S.nd[a + K++] = jlam;
        S.mk[a] = K;
        S.mr[a] = nrot;
        S.mf[a] = ndf;
    }
    g.sync();
    const int K = S.mk[a], nrot = S.mr[a];
    if (nrot > 0) {
        for (int i = t; i < nn; i += T) {
            const size_t row = (size_t)(a + i);
            for (int r = 0; r < nrot; ++r) {
                double* x = Z + row + (size_t)(a + S.ra[a + r]) * n;
                double* y = Z + row + (size_t)(a + S.rb[a + r]) * n;
                const double c_ = S.rc[a + r], s_ = S.rs[a + r];
                const double xi = *x, yi = *y;
                *x = c_ * xi + s_ * yi;
                *y = c_ * yi - s_ * xi;
            }
        }
    }
    for (int q = t; q < K; q += T) {
        S.dd[a + q] = S.ds[a + S.nd[a + q]];
        S.zz[a + q] = S.zs[a + S.nd[a + q]];
    }
}

// (t, T): this thread's rank among the T threads of the merge, each taking whole items;
// with R = WarpLanes, t and T count warps and the lanes of a warp share one item.
template <class R = SeqLanes>
__device__ void merge_roots(int t, int T, int a, int mid, const double* E, Scratch S, int* status,
                            R r = R{}) {
    const int K = S.mk[a];
    const double rho = 2.0 * fabs(E[mid - 1]);
    for (int j = t; j < K; j += T)
        secular_root(r, K, S.dd + a, S.zz + a, rho, j, S.org + a + j, S.tau + a + j, status);
}

// Gu-Eisenstat zhat
template <class R = SeqLanes>
__device__ void merge_zhat(int t, int T, int a, int mid, const double* E, Scratch S, R r = R{}) {
    const int K = S.mk[a];
    const double rho = 2.0 * fabs(E[mid - 1]);
    const double* dd = S.dd + a;
    const int* org = S.org + a;
    const double* tau = S.tau + a;
    for (int i = t; i < K; i += T) {
        double p = 1.0;
        for (int j = r.first(); j < K - 1; j += r.step())
            p *= (j < i) ? sec_delta(dd, org, tau, i, j) / (dd[i] - dd[j])
                         : sec_delta(dd, org, tau, i, j) / (dd[i] - dd[j + 1]);
        p = r.prod(p) * (-sec_delta(dd, org, tau, i, K - 1) / rho);
        if (r.leader()) S.zh[a + i] = copysign(sqrt(fmax(p, 0.0)), S.zz[a + i]);
    }
}

// eigenvectors of the rank-one problem (K x K at U[a.., a..], leading dim n)
template <class R = SeqLanes>
__device__ void merge_ucols(int t, int T, int a, int n, Scratch S, double* U, R r = R{}) {
    const int K = S.mk[a];
    const double* dd = S.dd + a;
    const int* org = S.org + a;
    const double* tau = S.tau + a;
    for (int j = t; j < K; j += T) {
        double nrm = 0.0;
        double* uc = U + (size_t)a + (size_t)(a + j) * n;
        for (int i = r.first(); i < K; i += r.step()) {
            const double u = S.zh[a + i] / sec_delta(dd, org, tau, i, j);
            uc[i] = u;
            nrm += u * u;
        }
        nrm = 1.0 / sqrt(r.sum(nrm));
        for (int i = r.first(); i < K; i += r.step()) uc[i] *= nrm;
    }
}

// the merged values in list order: nondeflated roots, then the deflated values
__device__ void merge_vals(int t, int T, int a, int b, Scratch S) {
    const int K = S.mk[a], nn = b - a;
    const double* dd = S.dd + a;
    const int* org = S.org + a;
    const double* tau = S.tau + a;
    for (int e = t; e < nn; e += T)
        S.vals[a + e] = e < K ? dd[org[e]] + tau[e] : S.ds[a + S.df[a + (e - K)]];
}

// final ascending order: nondeflated roots (list position j) then deflated values
// (list position K + q); ties keep list order
__device__ void merge_rank(int t, int T, int a, int b, Scratch S) {
    const int nn = b - a;
    for (int e = t; e < nn; e += T) {
        const double v = S.vals[a + e];
        int r = 0;
        for (int f = 0; f < nn; ++f) {
            const double w = S.vals[a + f];
            r += (w < v) || (w == v && f < e);
        }
        S.pos[a + e] = r;
    }
}

// deflated columns go to their final place in Qt
__device__ void merge_deflated(int t, int T, int a, int b, int n, const double* Z, double* Qt,
                               Scratch S) {
    const int nn = b - a, K = S.mk[a], ndf = S.mf[a];
    for (int e = t; e < nn * ndf; e += T) {
        const int i = e % nn, q = e / nn;
        const int src = a + S.perm[a + S.df[a + q]];
        Qt[(size_t)(a + i) + (size_t)(a + S.pos[a + K + q]) * n] = Z[(size_t)(a + i) + (size_t)src * n];
    }
}

__device__ void merge_copyback(int t, int T, int a, int b, int n, double* Z, double* D,
                               const double* Qt, Scratch S) {
    const int nn = b - a;
    for (int e = t; e < nn * nn; e += T) {
        const int i = e % nn, c = e / nn;
        Z[(size_t)(a + i) + (size_t)(a + c) * n] = Qt[(size_t)(a + i) + (size_t)(a + c) * n];
    }
    for (int e = t; e < nn; e += T) D[a + S.pos[a + e]] = S.vals[a + e];
}

// the whole merge inside one group
template <class G>
__device__ void dc_merge(G g, int a, int mid, int b, int n, double* Z, double* D,
                         const double* E, Scratch S, double* U, double* Qt, double* red,
                         double* gsm, int* status) {
    const int t = g.rank(), T = g.size();
    const int nn = b - a;
    const GroupLanes<kMergeLanes> gl{(int)(threadIdx.x & 31)};
    merge_prep(g, a, mid, b, n, Z, D, E, S, red);
    g.sync();
    merge_roots(t / kMergeLanes, T / kMergeLanes, a, mid, E, S, status, gl);
    g.sync();
    merge_zhat(t / kMergeLanes, T / kMergeLanes, a, mid, E, S, gl);
    g.sync();
    merge_ucols(t / kMergeLanes, T / kMergeLanes, a, n, S, U, gl);
    merge_vals(t, T, a, b, S);
    g.sync();
    merge_rank(t, T, a, b, S);
    g.sync();
    const int K = S.mk[a];
    if constexpr (std::is_same<G, BlockG>::value) {
        const int* perm = S.perm + a;
        const int* nd = S.nd + a;
        const int* pos = S.pos + a;
        auto fa = [=](int i, int k) -> double { return Z[(size_t)(a + i) + (size_t)(a + perm[nd[k]]) * n]; };
        auto fb = [=](int k, int j) -> double { return U[(size_t)(a + k) + (size_t)(a + j) * n]; };
        auto fc = [=](int i, int j) -> double& { return Qt[(size_t)(a + i) + (size_t)(a + pos[j]) * n]; };
        if (K > 0) nrg::cta_gemm(nn, K, K, 1.0, 0.0, fa, fb, fc, gsm);
    } else {
        for (int i = t; i < nn; i += T) {
            for (int j = 0; j < K; ++j) {
                double s = 0.0;
                for (int q = 0; q < K; ++q)
                    s += Z[(size_t)(a + i) + (size_t)(a + S.perm[a + S.nd[a + q]]) * n] *
                         U[(size_t)(a + q) + (size_t)(a + j) * n];
                Qt[(size_t)(a + i) + (size_t)(a + S.pos[a + j]) * n] = s;
            }
        }
    }
    merge_deflated(t, T, a, b, n, Z, Qt, S);
    g.sync();
    merge_copyback(t, T, a, b, n, Z, D, Qt, S);
    g.sync();
}

}  // namespace
