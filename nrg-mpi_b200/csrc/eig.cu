// Batched FP64 symmetric eigensolver for the symmetry-sector blocks of one NRG
// iteration (the dsyev('V','U') call of diagonalization.F90:267, one call per sector).
//
// One thread block owns one sector (sectors are queued largest first):
//   1. Householder tridiagonalisation of the lower triangle (H = Q T Q^T), reflectors
//      kept in the block's own storage;
//   2. divide and conquer on T (Cuppen tearing down to 1x1 leaves, deflation of small
//      z components and of close pole pairs by Givens rotations, secular roots by
//      bisection in coordinates shifted to the nearest pole, Gu-Eisenstat recomputation
//      of z for orthogonal eigenvectors); merges of up to 32 rows run one per warp,
//      larger merges use the whole block and an in-block tiled GEMM;
//   3. back-transformation V = Q Z with 32 reflectors at a time (compact WY form,
//      two in-block GEMMs per panel).
// Eigenvalues come out ascending with their eigenvectors in the same column order, as
// dsyev returns them.
#include "common.cuh"
#include "cta_gemm.cuh"

#include <cooperative_groups.h>
#include <math.h>
#include <type_traits>

namespace cg = cooperative_groups;

namespace {

constexpr int kThreads = 512;
constexpr int kNB = 32;          // reflectors per back-transform panel
constexpr double kEps = 1.1102230246251565e-16;

// ------------------------------------------------------------------------------------
// group abstraction: a whole block or one warp
// ------------------------------------------------------------------------------------
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

// secular equation g(t) = 1 + rho * sum zz_i^2 / ((dd_i - dd_o) - t)
__device__ double secular_g(int K, const double* dd, const double* zz, double rho, double base,
                            double t) {
    double s = 0.0;
    for (int i = 0; i < K; ++i) s += zz[i] * zz[i] / ((dd[i] - base) - t);
    return 1.0 + rho * s;
}

__device__ void secular_root(int K, const double* dd, const double* zz, double rho, int j,
                             int* org, double* tau, int* status) {
    double zsq = 0.0;
    for (int i = 0; i < K; ++i) zsq += zz[i] * zz[i];
    int o;
    double lo, hi;
    if (j < K - 1) {
        const double gap = dd[j + 1] - dd[j];
        const double fm = secular_g(K, dd, zz, rho, dd[j], 0.5 * gap);
        if (fm >= 0.0) { o = j; lo = 0.0; hi = 0.5 * gap; }
        else { o = j + 1; lo = -0.5 * gap; hi = 0.0; }
    } else {
        o = K - 1;
        const double up = rho * zsq;
        const double fm = secular_g(K, dd, zz, rho, dd[o], 0.5 * up);
        if (fm >= 0.0) { lo = 0.0; hi = 0.5 * up; } else { lo = 0.5 * up; hi = up; }
    }
    const double base = dd[o];
    double t = 0.5 * (lo + hi);
    int it = 0;
    for (; it < 200; ++it) {
        t = 0.5 * (lo + hi);
        if (t == lo || t == hi) break;
        const double gv = secular_g(K, dd, zz, rho, base, t);
        if (gv > 0.0) hi = t;
        else if (gv < 0.0) lo = t;
        else break;
    }
    if (!(t == t)) atomicOr(status, NRG_DEV_SECULAR);
    *org = o;
    *tau = t;
}

// dd_i - lambda_j
__device__ __forceinline__ double sec_delta(const double* dd, const int* org, const double* tau,
                                            int i, int j) {
    return (dd[i] - dd[org[j]]) - tau[j];
}

// ------------------------------------------------------------------------------------
// one merge of the divide and conquer: rows/cols [a, mid) and [mid, b) of Z (ld n)
// ------------------------------------------------------------------------------------
template <class G>
__device__ void dc_merge(G g, int a, int mid, int b, int n, double* Z, double* D,
                         const double* E, Scratch S, double* U, double* Qt, double* red,
                         double* gsm, int* status) {
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
        if (i < n1) {
            const double v = D[a + i];
            int lo = 0, hi = nn - n1;   // count of second-half values < v
            while (lo < hi) { int m = (lo + hi) >> 1; if (D[mid + m] < v) lo = m + 1; else hi = m; }
            rank = i + lo;
        } else {
            const double v = D[a + i];
            int lo = 0, hi = n1;        // count of first-half values <= v
            while (lo < hi) { int m = (lo + hi) >> 1; if (D[a + m] <= v) lo = m + 1; else hi = m; }
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
    // deflation (sequential scan, as dlaed2)
    if (t == 0) {
        int K = 0, ndf = 0, nrot = 0, jlam = -1;
        double* ds = S.ds + a;
        double* zs = S.zs + a;
        for (int j = 0; j < nn; ++j) {
            if (rho * fabs(zs[j]) <= tol) { S.df[a + ndf++] = j; continue; }
            if (jlam < 0) { jlam = j; continue; }
            double s_ = zs[jlam], c_ = zs[j];
            const double tau = hypot(c_, s_);
            const double tt = ds[j] - ds[jlam];
            c_ /= tau;
            s_ = -s_ / tau;
            if (fabs(tt * c_ * s_) <= tol) {
                zs[j] = tau;
                zs[jlam] = 0.0;
                S.ra[a + nrot] = S.perm[a + jlam];
                S.rb[a + nrot] = S.perm[a + j];
                S.rc[a + nrot] = c_;
                S.rs[a + nrot] = s_;
                ++nrot;
                const double tn = ds[jlam] * c_ * c_ + ds[j] * s_ * s_;
                ds[j] = ds[jlam] * s_ * s_ + ds[j] * c_ * c_;
                ds[jlam] = tn;
                S.df[a + ndf++] = jlam;
                jlam = j;
            } else {
                S.nd[a + K++] = jlam;
                jlam = j;
            }
        }
        if (jlam >= 0) S.nd[a + K++] = jlam;
        S.mk[a] = K;
        S.mr[a] = nrot;
        S.mf[a] = ndf;
    }
    g.sync();
    const int K = S.mk[a], nrot = S.mr[a], ndf = S.mf[a];
    // apply the deflation rotations, in order, row by row
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
    g.sync();
    const double* dd = S.dd + a;
    const double* zz = S.zz + a;
    int* org = S.org + a;
    double* tau = S.tau + a;
    for (int j = t; j < K; j += T) secular_root(K, dd, zz, rho, j, org + j, tau + j, status);
    g.sync();
    // Gu-Eisenstat zhat
    for (int i = t; i < K; i += T) {
        double p = -sec_delta(dd, org, tau, i, K - 1) / rho;
        for (int j = 0; j < i; ++j) p *= sec_delta(dd, org, tau, i, j) / (dd[i] - dd[j]);
        for (int j = i; j < K - 1; ++j) p *= sec_delta(dd, org, tau, i, j) / (dd[i] - dd[j + 1]);
        S.zh[a + i] = copysign(sqrt(fmax(p, 0.0)), zz[i]);
    }
    g.sync();
    // eigenvectors of the rank-one problem: U(:, j), K x K, stored at U[a.., a..] (ld n)
    for (int j = t; j < K; j += T) {
        double nrm = 0.0;
        double* uc = U + (size_t)a + (size_t)(a + j) * n;
        for (int i = 0; i < K; ++i) {
            const double u = S.zh[a + i] / sec_delta(dd, org, tau, i, j);
            uc[i] = u;
            nrm += u * u;
        }
        nrm = 1.0 / sqrt(nrm);
        for (int i = 0; i < K; ++i) uc[i] *= nrm;
    }
    // final ascending order: nondeflated roots (list position j) then deflated values
    // (list position K + q); ties keep list order
    for (int e = t; e < nn; e += T) {
        const double v = e < K ? dd[org[e]] + tau[e] : S.ds[a + S.df[a + (e - K)]];
        S.vals[a + e] = v;
    }
    g.sync();
    for (int e = t; e < nn; e += T) {
        const double v = S.vals[a + e];
        int r = 0;
        for (int f = 0; f < nn; ++f) {
            const double w = S.vals[a + f];
            r += (w < v) || (w == v && f < e);
        }
        S.pos[a + e] = r;
    }
    g.sync();
    // Qt(:, pos) = Z(:, nondeflated cols) * U  |  Z(:, deflated col)
    if constexpr (std::is_same<G, BlockG>::value) {
        const int* perm = S.perm + a;
        const int* nd = S.nd + a;
        const int* pos = S.pos + a;
        auto fa = [=](int i, int k) -> double {
            return Z[(size_t)(a + i) + (size_t)(a + perm[nd[k]]) * n];
        };
        auto fb = [=](int k, int j) -> double { return U[(size_t)(a + k) + (size_t)(a + j) * n]; };
        auto fc = [=](int i, int j) -> double& {
            return Qt[(size_t)(a + i) + (size_t)(a + pos[j]) * n];
        };
        if (K > 0) nrg::cta_gemm(nn, K, K, 1.0, 0.0, fa, fb, fc, gsm);
        for (int e = t; e < nn * ndf; e += T) {
            const int i = e % nn, q = e / nn;
            const int src = a + S.perm[a + S.df[a + q]];
            Qt[(size_t)(a + i) + (size_t)(a + S.pos[a + K + q]) * n] = Z[(size_t)(a + i) + (size_t)src * n];
        }
    } else {
        // warp: nn <= 32, each lane one row
        for (int i = t; i < nn; i += T) {
            for (int j = 0; j < K; ++j) {
                double s = 0.0;
                for (int q = 0; q < K; ++q)
                    s += Z[(size_t)(a + i) + (size_t)(a + S.perm[a + S.nd[a + q]]) * n] *
                         U[(size_t)(a + q) + (size_t)(a + j) * n];
                Qt[(size_t)(a + i) + (size_t)(a + S.pos[a + j]) * n] = s;
            }
            for (int q = 0; q < ndf; ++q) {
                const int src = a + S.perm[a + S.df[a + q]];
                Qt[(size_t)(a + i) + (size_t)(a + S.pos[a + K + q]) * n] = Z[(size_t)(a + i) + (size_t)src * n];
            }
        }
    }
    g.sync();
    for (int e = t; e < nn * nn; e += T) {
        const int i = e % nn, c = e / nn;
        Z[(size_t)(a + i) + (size_t)(a + c) * n] = Qt[(size_t)(a + i) + (size_t)(a + c) * n];
    }
    for (int e = t; e < nn; e += T) D[a + S.pos[a + e]] = S.vals[a + e];
    g.sync();
}

// ------------------------------------------------------------------------------------
// the per-sector kernel
// ------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_syev(const SyevSector* __restrict__ secs,
                                                    double* __restrict__ eigbuf,
                                                    double* __restrict__ evals,
                                                    double* __restrict__ wsd, int* __restrict__ wsi,
                                                    int* status) {
    extern __shared__ double sm[];
    const SyevSector sec = secs[blockIdx.x];
    const int n = sec.n;
    const int tid = threadIdx.x, T = blockDim.x;
    double* A = eigbuf + sec.a_off;
    double* ev = evals + sec.e_off;
    if (n == 1) {
        if (tid == 0) { ev[0] = A[0]; A[0] = 1.0; }
        return;
    }
    // workspace
    double* W = wsd + sec.w_off;
    const long long sq = (long long)n * n;
    double* Z = W;
    double* U = W + sq;
    double* Qt = W + 2 * sq;
    const long long qt = sq > 64LL * n ? sq : 64LL * n;
    double* vec = W + 2 * sq + qt;
    double* Dd = vec;           // n : diagonal / eigenvalues
    double* Ee = vec + n;       // n : off-diagonal
    double* TAU = vec + 2 * n;  // n : reflector scalars
    Scratch S;
    S.z = vec + 3 * n; S.ds = vec + 4 * n; S.zs = vec + 5 * n; S.dd = vec + 6 * n;
    S.zz = vec + 7 * n; S.tau = vec + 8 * n; S.zh = vec + 9 * n; S.vals = vec + 10 * n;
    S.rc = vec + 11 * n; S.rs = vec + 12 * n;
    int* I = wsi + sec.i_off;
    S.perm = I; S.nd = I + n; S.df = I + 2 * n; S.org = I + 3 * n; S.pos = I + 4 * n;
    S.ra = I + 5 * n; S.rb = I + 6 * n; S.mk = I + 7 * n; S.mr = I + 8 * n; S.mf = I + 9 * n;

    double* red = sm;                 // 32
    double* gsm = sm + 32;            // gemm staging: 16*(4*T/16+1) + 16*65
    const int gsz = 16 * (4 * (T / 16) + 1) + 16 * 65;
    double* vs = sm + 32 + gsz;       // n
    double* ps = vs + n;              // n

    // ---- 1. tridiagonalisation (lower, full storage kept symmetric) ----
    for (int k = 0; k < n - 1; ++k) {
        const int m = n - k - 1;
        double* col = A + (size_t)k * n;
        const double alpha = col[k + 1];
        double part = 0.0;
        for (int i = k + 2 + tid; i < n; i += T) part += col[i] * col[i];
        const double xn2 = block_sum(part, red);
        if (xn2 == 0.0) {
            if (tid == 0) { Ee[k] = alpha; TAU[k] = 0.0; }
            continue;
        }
        const double beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
        const double tt = (beta - alpha) / beta;
        const double scal = 1.0 / (alpha - beta);
        for (int i = tid; i < m; i += T) {
            double vi = 1.0;
            if (i > 0) { vi = col[k + 1 + i] * scal; col[k + 1 + i] = vi; }
            vs[i] = vi;
        }
        if (tid == 0) { Ee[k] = beta; TAU[k] = tt; }
        __syncthreads();
        double pv_part = 0.0;
        for (int i = tid; i < m; i += T) {
            const double* Ai = A + (size_t)(k + 1 + i) + (size_t)(k + 1) * n;
            double s0 = 0.0, s1 = 0.0;
            int j = 0;
            for (; j + 1 < m; j += 2) {
                s0 = fma(Ai[(size_t)j * n], vs[j], s0);
                s1 = fma(Ai[(size_t)(j + 1) * n], vs[j + 1], s1);
            }
            if (j < m) s0 = fma(Ai[(size_t)j * n], vs[j], s0);
            const double pi = tt * (s0 + s1);
            ps[i] = pi;
            pv_part += pi * vs[i];
        }
        const double pv = block_sum(pv_part, red);
        const double h = -0.5 * tt * pv;
        for (int i = tid; i < m; i += T) ps[i] += h * vs[i];
        __syncthreads();
        for (int j = 0; j < m; ++j) {
            const double vj = vs[j], wj = ps[j];
            double* Aj = A + (size_t)(k + 1) + (size_t)(k + 1 + j) * n;
            for (int i = tid; i < m; i += T) Aj[i] -= vs[i] * wj + ps[i] * vj;
        }
        __syncthreads();
    }
    for (int k = tid; k < n; k += T) Dd[k] = A[(size_t)k + (size_t)k * n];
    if (tid == 0) Ee[n - 1] = 0.0;
    __syncthreads();

    // ---- 2. divide and conquer on (Dd, Ee) -> eigenvalues in Dd, vectors in Z ----
    for (long long e = tid; e < sq; e += T) Z[e] = 0.0;
    __syncthreads();
    for (int i = tid; i < n; i += T) {
        Z[(size_t)i + (size_t)i * n] = 1.0;
        double dv = Dd[i];
        if (i > 0) dv -= fabs(Ee[i - 1]);
        if (i < n - 1) dv -= fabs(Ee[i]);
        S.vals[i] = dv;
    }
    __syncthreads();
    for (int i = tid; i < n; i += T) Dd[i] = S.vals[i];
    __syncthreads();
    const int warp = tid >> 5, lane = tid & 31, nwarps = T >> 5;
    for (int s = 1; s < n; s *= 2) {
        if (2 * s <= 32) {
            WarpG wg{lane};
            int mi = 0;
            for (int a = 0; a + s < n; a += 2 * s, ++mi) {
                if (mi % nwarps != warp) continue;
                const int mid = a + s, b = min(a + 2 * s, n);
                dc_merge(wg, a, mid, b, n, Z, Dd, Ee, S, U, Qt, red, gsm, status);
            }
            __syncthreads();
        } else {
            BlockG bg;
            for (int a = 0; a + s < n; a += 2 * s) {
                const int mid = a + s, b = min(a + 2 * s, n);
                dc_merge(bg, a, mid, b, n, Z, Dd, Ee, S, U, Qt, red, gsm, status);
            }
        }
    }
    __syncthreads();

    // ---- 3. back-transformation Z <- Q Z, panels of kNB reflectors, last first ----
    const int nr = n - 1;
    double* Ts = vs;   // kNB x kNB (smem reuse of the tridiagonalisation vectors)
    double* Gs = vs + kNB * kNB;
    for (int jb = ((nr - 1) / kNB) * kNB; jb >= 0; jb -= kNB) {
        const int b = min(kNB, nr - jb);
        const int r0 = jb + 1, mr = n - r0;
        double* Vb = U;  // mr x b, ld mr
        for (long long e = tid; e < (long long)mr * b; e += T) {
            const int i = (int)(e % mr), c = (int)(e / mr);
            const int k = jb + c, row = r0 + i;
            double v = 0.0;
            if (row == k + 1) v = 1.0;
            else if (row > k + 1) v = A[(size_t)row + (size_t)k * n];
            Vb[e] = v;
        }
        __syncthreads();
        for (int e = tid; e < b * b; e += T) {
            const int p = e % b, q = e / b;
            double s = 0.0;
            if (p < q) {
                const double* vp = Vb + (size_t)p * mr;
                const double* vq = Vb + (size_t)q * mr;
                for (int i = 0; i < mr; ++i) s = fma(vp[i], vq[i], s);
            }
            Gs[p + q * kNB] = s;
            Ts[p + q * kNB] = 0.0;
        }
        __syncthreads();
        if (warp == 0) {
            for (int c = 0; c < b; ++c) {
                const double tc = TAU[jb + c];
                // y_q = -tc * G(q, c), q < c; T(p, c) = sum_{q=p}^{c-1} T(p, q) y_q
                double acc = 0.0;
                if (lane < c) {
                    for (int q = lane; q < c; ++q) acc += Ts[lane + q * kNB] * (-tc * Gs[q + c * kNB]);
                }
                __syncwarp();
                if (lane < c) Ts[lane + c * kNB] = acc;
                if (lane == 0) Ts[c + c * kNB] = tc;
                __syncwarp();
            }
        }
        __syncthreads();
        // Wm = Vb^T Z(r0:, :)   (b x n, ld b) in Qt
        double* Wm = Qt;
        double* W2 = Qt + (size_t)kNB * n;
        {
            auto fa = [=](int i, int k) -> double { return Vb[(size_t)k + (size_t)i * mr]; };
            auto fb = [=](int k, int j) -> double { return Z[(size_t)(r0 + k) + (size_t)j * n]; };
            auto fc = [=](int i, int j) -> double& { return Wm[(size_t)i + (size_t)j * b]; };
            nrg::cta_gemm(b, n, mr, 1.0, 0.0, fa, fb, fc, gsm);
        }
        __syncthreads();
        for (long long e = tid; e < (long long)b * n; e += T) {
            const int p = (int)(e % b);
            const long long j = e / b;
            double s = 0.0;
            for (int q = p; q < b; ++q) s = fma(Ts[p + q * kNB], Wm[(size_t)q + (size_t)j * b], s);
            W2[e] = s;
        }
        __syncthreads();
        {
            auto fa = [=](int i, int k) -> double { return Vb[(size_t)i + (size_t)k * mr]; };
            auto fb = [=](int k, int j) -> double { return W2[(size_t)k + (size_t)j * b]; };
            auto fc = [=](int i, int j) -> double& { return Z[(size_t)(r0 + i) + (size_t)j * n]; };
            nrg::cta_gemm(mr, n, b, -1.0, 1.0, fa, fb, fc, gsm);
        }
        __syncthreads();
    }
    // ---- outputs: eigenvalues, eigenvectors (into the block's own storage) ----
    for (int i = tid; i < n; i += T) ev[i] = Dd[i];
    for (long long e = tid; e < sq; e += T) A[e] = Z[e];
}

}  // namespace

int launch_syev(const SyevSector* d_secs, int nsec, int max_n, double* eigbuf, double* evals,
                double* wsd, int* wsi, int* d_status, cudaStream_t st) {
    if (nsec == 0) return NRG_OK;
    const int gsz = 16 * (4 * (kThreads / 16) + 1) + 16 * 65;
    size_t smem = sizeof(double) * (32 + gsz + 2 * (size_t)(max_n > kNB * kNB ? max_n : kNB * kNB) + kNB * kNB);
    if (smem > 227 * 1024) {
        nrg_set_error_message("sector of order %d exceeds the shared-memory plan", max_n);
        return NRG_ERR_TOO_LARGE;
    }
    static size_t configured = 0;
    if (smem > 48 * 1024 && smem > configured) {
        NRG_CUDA_TRY(cudaFuncSetAttribute(k_syev, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        configured = smem;
    }
    k_syev<<<nsec, kThreads, smem, st>>>(d_secs, eigbuf, evals, wsd, wsi, d_status);
    NRG_CUDA_TRY(cudaGetLastError());
    return NRG_OK;
}
