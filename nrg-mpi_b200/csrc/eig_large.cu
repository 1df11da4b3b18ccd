// FP64 eigensolver for the large symmetry sectors of one iteration (order > 128), spread
// over the whole GPU instead of one block per sector.  All large sectors advance together:
//   1. blocked Householder tridiagonalisation (panels of 32 columns, the dlatrd scheme):
//      per column one block per sector updates the column with the pending panel
//      reflectors and forms the Householder vector, then a many-block kernel computes the
//      symmetric matrix-vector product with the trailing matrix (column dot products,
//      coalesced); after each panel the trailing matrix takes the rank-64 update
//      A -= [V W][W V]^T as one grouped GEMM;
//   2. divide and conquer: merges up to 128 rows inside one block per sector; larger
//      merges in phases (deflation, secular roots, Gu-Eisenstat z, rank-one eigenvectors,
//      final order) with the eigenvector update Z(:, kept) * U as a grouped GEMM;
//   3. back-transformation in panels of 64 reflectors: Gram matrix and V^T Z as grouped
//      GEMMs, the triangular factor T in one block, then Z -= (V T)(V^T Z).
#include "eig_common.cuh"
#include "internal.hpp"

#include <cooperative_groups.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace cg = cooperative_groups;

namespace {

constexpr int NB = 32;        // tridiagonalisation panel
constexpr int NBB = 64;       // back-transformation panel
constexpr int DC_LOW = 128;   // merges of up to this many rows run inside one block
constexpr int TPB = 256;
constexpr int CB = 32;        // columns per block in the symmetric matrix-vector product
constexpr int kTriCL = 8;     // blocks per cluster of the one-launch tridiagonalisation
constexpr int kTriCL16Min = 1 << 30;   // order from which a launch takes 16-block clusters

struct LSec {
    long long a_off, e_off, w_off, i_off;
    int n, pad;
};

// workspace per sector: Z, U, Qt (n x n each), the panel V | W (n x 2 NB), y, the D&C
// vectors (16 n + 64), then the back-transformation's T factors and explicit reflector
// panels ((n + NBB)^2 bounds both)
long long lws_doubles(long long n) {
    return 3 * n * n + 2LL * NB * n + n + 16 * n + 64 + (n + NBB) * (n + NBB);
}
long long lws_ints(long long n) { return 12 * n + 64; }

struct LView {
    double *A, *Z, *U, *Qt, *VW, *y, *vec, *D, *E, *TAU, *R;
    int* I;
    Scratch S;
    int n;
};

__device__ LView lview(const LSec& s, double* eigbuf, double* wsd, int* wsi) {
    LView v;
    const long long n = s.n, sq = n * n;
    v.n = s.n;
    v.A = eigbuf + s.a_off;
    double* W = wsd + s.w_off;
    v.Z = W;
    v.U = W + sq;
    v.Qt = W + 2 * sq;
    v.VW = W + 3 * sq;
    v.y = v.VW + 2LL * NB * n;
    v.vec = v.y + n;
    v.D = v.vec;
    v.E = v.vec + n;
    v.TAU = v.vec + 2 * n;
    v.R = v.vec + 16 * n + 64;
    v.I = wsi + s.i_off;
    v.S = scratch_at(v.vec, v.I, s.n);
    return v;
}

// ---------------------------------------------------------------------------------
// tridiagonalisation
// ---------------------------------------------------------------------------------

// W(:, jj) for column c of the panel (rows c+1..n-1): dlatrd's w update
__device__ void finish_w(LView& L, int c, int jj, const double* t1s, double* t1, double* t2, double* red) {
    (void)t1s;
    const int n = L.n, tid = threadIdx.x, T = blockDim.x;
    const int warp = tid >> 5, lane = tid & 31, nw = T >> 5;
    const double* V = L.VW;
    double* W = L.VW + (size_t)NB * n;
    const double* v = V + (size_t)jj * n;
    for (int q = warp; q < 2 * jj; q += nw) {
        const double* col = q < jj ? W + (size_t)q * n : V + (size_t)(q - jj) * n;
        double s = 0.0;
        for (int i = c + 1 + lane; i < n; i += 32) s = fma(col[i], v[i], s);
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) { if (q < jj) t1[q] = s; else t2[q - jj] = s; }
    }
    __syncthreads();
    const double tau = L.TAU[c];
    double* w = W + (size_t)jj * n;
    double part = 0.0;
    for (int i = c + 1 + tid; i < n; i += T) {
        double s = L.y[i];
        for (int q = 0; q < jj; ++q) s -= V[i + (size_t)q * n] * t1[q] + W[i + (size_t)q * n] * t2[q];
        s *= tau;
        w[i] = s;
        part += s * v[i];
    }
    const double wv = block_sum(part, red);
    const double al = -0.5 * tau * wv;
    for (int i = c + 1 + tid; i < n; i += T) w[i] += al * v[i];
    __syncthreads();
}

__global__ void __launch_bounds__(TPB) k_tri_col(const LSec* __restrict__ secs, int k, double* eigbuf,
                                                 double* wsd, int* wsi) {
    __shared__ double red[32];
    __shared__ double t1[NB], t2[NB];
    const LSec sec = secs[blockIdx.x];
    if (k > sec.n - 2) return;
    LView L = lview(sec, eigbuf, wsd, wsi);
    const int n = L.n, tid = threadIdx.x, T = blockDim.x;
    const int j = k % NB;
    if (j > 0) finish_w(L, k - 1, j - 1, nullptr, t1, t2, red);
    double* V = L.VW;
    double* W = L.VW + (size_t)NB * n;
    double* col = L.A + (size_t)k * n;
    // column k takes the pending updates of the panel's first j reflectors
    for (int i = k + tid; i < n; i += T) {
        double s = 0.0;
        for (int q = 0; q < j; ++q)
            s += V[i + (size_t)q * n] * W[k + (size_t)q * n] + W[i + (size_t)q * n] * V[k + (size_t)q * n];
        col[i] -= s;
    }
    __syncthreads();
    if (tid == 0) L.D[k] = col[k];
    const double alpha = col[k + 1];
    double part = 0.0;
    for (int i = k + 2 + tid; i < n; i += T) part += col[i] * col[i];
    const double xn2 = block_sum(part, red);
    double* v = V + (size_t)j * n;
    if (xn2 == 0.0) {
        for (int i = k + 1 + tid; i < n; i += T) v[i] = (i == k + 1) ? 1.0 : 0.0;
        if (tid == 0) { L.E[k] = alpha; L.TAU[k] = 0.0; }
        return;
    }
    const double beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
    const double tt = (beta - alpha) / beta;
    const double scal = 1.0 / (alpha - beta);
    for (int i = k + 1 + tid; i < n; i += T) {
        double vi = 1.0;
        if (i > k + 1) { vi = col[i] * scal; col[i] = vi; }
        v[i] = vi;
    }
    if (tid == 0) { L.E[k] = beta; L.TAU[k] = tt; }
}

// y(i) = sum_{l > k} A(l, i) v(l) for i > k: one warp per column, CB columns per block
__global__ void __launch_bounds__(TPB) k_tri_symv(const LSec* __restrict__ secs, int nsec, int k,
                                                  double* eigbuf, double* wsd, int* wsi) {
    extern __shared__ double vsm[];
    // find this block's sector among those still active at column k
    int s = 0, base = 0;
    for (; s < nsec; ++s) {
        const int n = secs[s].n;
        if (k > n - 2) continue;
        const int nb = (n - k - 1 + CB - 1) / CB;
        if ((int)blockIdx.x < base + nb) break;
        base += nb;
    }
    if (s >= nsec) return;
    LView L = lview(secs[s], eigbuf, wsd, wsi);
    const int n = L.n, m = n - k - 1;
    const int j = k % NB;
    const double* v = L.VW + (size_t)j * n + (k + 1);
    for (int i = threadIdx.x; i < m; i += blockDim.x) vsm[i] = v[i];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int c0 = ((int)blockIdx.x - base) * CB;
    for (int cc = warp; cc < CB; cc += nw) {
        const int ci = c0 + cc;
        if (ci >= m) break;
        const double* col = L.A + (size_t)(k + 1 + ci) * n + (k + 1);
        double s0 = 0.0, s1 = 0.0;
        int l = lane;
        for (; l + 32 < m; l += 64) {
            s0 = fma(col[l], vsm[l], s0);
            s1 = fma(col[l + 32], vsm[l + 32], s1);
        }
        if (l < m) s0 = fma(col[l], vsm[l], s0);
        double sum = s0 + s1;
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        if (lane == 0) L.y[k + 1 + ci] = sum;
    }
}

// W for the last column a sector processed in the panel starting at p
__global__ void __launch_bounds__(TPB) k_tri_finish(const LSec* __restrict__ secs, int p, double* eigbuf,
                                                    double* wsd, int* wsi) {
    __shared__ double red[32];
    __shared__ double t1[NB], t2[NB];
    const LSec sec = secs[blockIdx.x];
    const int c = min(p + NB - 1, sec.n - 2);
    if (c < p) return;
    LView L = lview(sec, eigbuf, wsd, wsi);
    finish_w(L, c, c - p, nullptr, t1, t2, red);
}

// ---------------------------------------------------------------------------------
// tridiagonalisation by one thread-block cluster per sector
// ---------------------------------------------------------------------------------
// The same panel scheme (dlatrd) in one launch.  The CL blocks of a cluster split the
// indices of the sector cyclically (index i belongs to block i % CL, as a row and as a
// column) and keep the panel rows V(i, :), W(i, :) of their own indices in shared
// memory.  Two cluster barriers per column k:
//   A  each block updates its rows of column k with the pending panel reflectors (read
//      as row k of its own columns: the trailing matrix is stored in full) and stores
//      them into the shared memory of every block of the cluster, with its partial
//      |x|^2; barrier 1; every block now holds the whole column and forms the same
//      beta, tau and Householder vector v;
//   B  y(l) = A(:, l) . v for the own columns l (coalesced column reads), partial
//      W^T v, V^T v over the own rows and partial y . v are stored into every block;
//      the owner of row k+1 also sends its panel row and y(k+1); barrier 2; every block
//      forms t1 = W^T v, t2 = V^T v, w.v = tau (y.v - 2 t1.t2) and
//      w = tau (y - V t1 - W t2) - (tau/2)(w.v) v for its own rows, and the pivot row's
//      w for the next column.
// After each panel every block writes its panel rows of V and W, the reflectors and the
// panel's D, E and tau to global memory (inside the panel they stay in shared memory: a
// global store pending at a cluster barrier makes the barrier wait for it) and applies
// A -= V W^T + W V^T to its own columns.  Blocks of different clusters never touch each
// other's data.
constexpr int TT = 512;     // threads per block of the cluster kernel
constexpr int TRW = 128;    // rows per staged chunk of the trailing update
constexpr int P2W = 2 * NB + 2;   // partials per block: W^T v | V^T v | y.v

struct TriLayout {
    int MM, PN, NRB;   // own indices per block, rows (even), row batches of 512 (rounded up)
    __host__ __device__ long long doubles(int CL) const {
        // the panel rows AR share their space with the staging of the trailing update; v
        // for the product (PN + 2, 16-byte aligned) last
        const long long stage = (long long)NB * MM > 2LL * NB * TRW ? (long long)NB * MM : 2LL * NB * TRW;
        return 2LL * NB * MM + PN + MM + (long long)CL * P2W + CL + 2 + 2LL * NB + 2LL * NB + P2W + 32 +
               stage + (long long)NRB * MM + 3LL * NB + PN + 4;
    }
};

// the sums over the warp of four values: lane l ends with the total of value (l >> 3) & 3
// (every lane of a group of eight with the same bits), by halving exchanges
__device__ __forceinline__ double warp_sum4(double a0, double a1, double a2, double a3, int lane) {
    const bool h16 = lane & 16, h8 = lane & 8;
    double k0 = h16 ? a2 : a0, k1 = h16 ? a3 : a1;
    k0 += __shfl_xor_sync(0xffffffffu, h16 ? a0 : a2, 16);
    k1 += __shfl_xor_sync(0xffffffffu, h16 ? a1 : a3, 16);
    double kk = h8 ? k1 : k0;
    kk += __shfl_xor_sync(0xffffffffu, h8 ? k0 : k1, 8);
    kk += __shfl_xor_sync(0xffffffffu, kk, 4);
    kk += __shfl_xor_sync(0xffffffffu, kk, 2);
    kk += __shfl_xor_sync(0xffffffffu, kk, 1);
    return kk;
}

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// w = tau (y - sum_q (V_q t1_q + W_q t2_q)) + al v with explicit roundings, so that every
// block computes the pivot row's w bit-identically to its owner (two partial sums)
__device__ __forceinline__ double w_entry(double y, const double* Vr, const double* Wr, int stride,
                                          const double* t1, const double* t2, int j, double tau,
                                          double al, double v) {
    double s = y, s2 = 0.0;
    #pragma unroll 4
    for (int q = 0; q < j; ++q) {
        s = fma(-Vr[q * stride], t1[q], s);
        s2 = fma(-Wr[q * stride], t2[q], s2);
    }
    return fma(al, v, __dmul_rn(tau, __dadd_rn(s, s2)));
}

template <int CL>
__global__ void __launch_bounds__(TT, 1) k_tri_cluster(const LSec* __restrict__ secs, TriLayout lay,
                                                      double* eigbuf, double* wsd, int* wsi) {
    extern __shared__ double sm[];
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    const LSec sec = secs[blockIdx.x / CL];
    LView L = lview(sec, eigbuf, wsd, wsi);
    const int n = L.n, MM = lay.MM;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = TT / 32;
    double* VO = sm;                       // NB x MM: V(own row m, q) at q*MM + m
    double* WO = VO + (size_t)NB * MM;     // NB x MM
    double* cv = WO + (size_t)NB * MM;     // column k (rows > k), then v, by row
    double* ys = cv + lay.PN;              // y of the own columns
    double* P2 = ys + MM;                  // CL x P2W partials, by source block
    double* redA = P2 + CL * P2W;          // CL partial |x|^2
    double* Y1 = redA + CL;                // y(k+1) from its owner (2 slots)
    double* pivn = Y1 + 2;                 // 2 NB: V(k+1, q) | W(k+1, q) from its owner
    double* piv = pivn + 2 * NB;           // 2 NB: W(k, q) | V(k, q) of the current pivot row
    double* tsum = piv + 2 * NB;           // t1 | t2 | y.v
    double* red = tsum + P2W;              // 32
    double* AR = red + 32;                 // NB x MM: A(p + q, own column m), during the columns
    double* stV = AR;                      // NB x TRW staged rows of V (transposed), during the
    double* stW = stV + NB * TRW;          // trailing update; NB x TRW
    double* ysp = AR + ((size_t)NB * MM > 2 * NB * TRW ? (size_t)NB * MM : 2 * NB * TRW);   // NRB x MM
    double* pan = ysp + (size_t)lay.NRB * MM;   // D | E | tau of the panel's columns
    // v of the current column for the product, row r at vv[r + par]: with par the parity
    // of the own columns' offsets, rows pair up on 16-byte boundaries in A and in vv
    double* vv = sm + ((pan - sm + 3 * NB + 1) & ~(ptrdiff_t)1);
    double* Vg = L.VW;
    double* Wg = L.VW + (size_t)NB * n;
    double* A = L.A;
    const int cnt = (n - rank + CL - 1) / CL;                           // own indices rank + CL*m
    auto first_own = [&](int i0) { return (i0 - rank + CL - 1) / CL; };  // i0 >= 0
    // CL is even, so every own column's offset (rank + CL m) n has the parity of rank n
    const int par = (int)(((reinterpret_cast<uintptr_t>(A) >> 3) + (uintptr_t)rank * n) & 1);

    for (int p = 0; p < n - 1; p += NB) {
        const int last = min(p + NB - 1, n - 2);
        const int jn = last - p + 1;
        // rows p..last of the own columns: the panel's columns read them as rows (the
        // trailing matrix is stored in full) and nothing writes them during the panel
        {
            const int m0 = first_own(p);
            for (int e = tid; e < jn * (cnt - m0); e += TT) {
                const int q = e % jn, m = m0 + e / jn;
                AR[q * MM + m] = __ldcg(A + (size_t)(p + q) + (size_t)(rank + CL * m) * n);
            }
            __syncthreads();
        }
        for (int k = p; k <= last; ++k) {
            const int j = k - p;
            // ---- A: own rows of column k, broadcast ----
            const int m = first_own(k) + tid;
            const bool act = m < cnt;
            const int i = rank + CL * m;
            double c = 0.0, ss = 0.0;
            if (act) {
                double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
                int q = 0;
                #pragma unroll 4
                for (; q + 1 < j; q += 2) {
                    s0 = fma(VO[q * MM + m], piv[q], s0);
                    s1 = fma(WO[q * MM + m], piv[NB + q], s1);
                    s2 = fma(VO[(q + 1) * MM + m], piv[q + 1], s2);
                    s3 = fma(WO[(q + 1) * MM + m], piv[NB + q + 1], s3);
                }
                if (q < j) {
                    s0 = fma(VO[q * MM + m], piv[q], s0);
                    s1 = fma(WO[q * MM + m], piv[NB + q], s1);
                }
                c = AR[j * MM + m] - ((s0 + s2) + (s1 + s3));
                if (i == k) pan[j] = c;
                if (i >= k + 2) ss = c * c;
                if (i >= k + 1)
                    for (int r = 0; r < CL; ++r) cluster.map_shared_rank(cv, r)[i] = c;
            }
            const double ssb = block_sum(ss, red);
            if (tid < CL) cluster.map_shared_rank(redA, tid)[rank] = ssb;
            cluster.sync();
            double xn2 = 0.0;
            for (int r = 0; r < CL; ++r) xn2 += redA[r];
            const double alpha = cv[k + 1];
            double beta = alpha, tau = 0.0, scal = 0.0;
            if (xn2 != 0.0) {
                beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
                tau = (beta - alpha) / beta;
                scal = 1.0 / (alpha - beta);
            }
            // v into vv (cv(k+1) keeps alpha, which every thread reads above): v(k+1) = 1, and
            // the row before it 0 for a product that starts one row early to pair the rows
            for (int r = k + 2 + tid; r < n; r += TT) vv[r + par] = xn2 == 0.0 ? 0.0 : cv[r] * scal;
            if (tid == 0) { vv[k + par] = 0.0; vv[k + 1 + par] = 1.0; }
            if (act && i >= k + 1) VO[j * MM + m] = (i == k + 1) ? 1.0 : (xn2 == 0.0 ? 0.0 : c * scal);
            if (tid == 0) { pan[NB + j] = beta; pan[2 * NB + j] = tau; }
            __syncthreads();
            // ---- B: partial W^T v, V^T v over the own rows, the next pivot row, then y of
            // the own columns and partial y.v ----
            const int mB = first_own(k + 1);
            // the product's rows start at rs = k + 1 or k (vv(k) = 0), so that the offsets of
            // (rs, rs + 1) in A and in vv are even
            const int rs = (k + 1) - ((k + 1 + par) & 1);
            const int nq = (cnt - mB + 3) / 4, nrb = (n - rs + 511) / 512, nitems = nq * nrb;
            const double* vj = VO + j * MM;
            const bool pivot_owner = (rank == (k + 1) % CL);
            if (pivot_owner && k + 1 <= last) {
                for (int e = tid; e < 2 * j * CL; e += TT) {
                    const int q = e / CL, r = e % CL;
                    const double val = q < j ? VO[q * MM + mB] : WO[(q - j) * MM + mB];
                    cluster.map_shared_rank(pivn, r)[q < j ? q : NB + (q - j)] = val;
                }
            }
            // the 2j partial dots over the own rows, four per warp (o = 4 g + c: W^T v for
            // o < j, V^T v after), one exchange reduction for the four
            for (int g = warp; 4 * g < 2 * j; g += NW) {
                const double* colp[4];
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const int o = min(4 * g + c, 2 * j - 1);
                    colp[c] = (o < j) ? WO + o * MM : VO + (o - j) * MM;
                }
                double s4[4] = {0.0, 0.0, 0.0, 0.0};
                for (int mm = mB + lane; mm < cnt; mm += 32) {
                    const double vm = vj[mm];
#pragma unroll
                    for (int c = 0; c < 4; ++c) s4[c] = fma(colp[c][mm], vm, s4[c]);
                }
                const double tot = warp_sum4(s4[0], s4[1], s4[2], s4[3], lane);
                const int o = 4 * g + ((lane >> 3) & 3);
                if (o < 2 * j)
                    for (int r = lane & 7; r < CL; r += 8)
                        cluster.map_shared_rank(P2, r)[rank * P2W + (o < j ? o : NB + (o - j))] = tot;
            }
            // y = A v in work items of four own columns x 512 rows (256 row pairs), one warp
            // each: 16-byte loads of row pairs, eight pairs per lane and column in two
            // batches of 16 loads, bounds checked only in the last row batch; one exchange
            // reduction of the four sums per item; partial sums per row batch, added in a
            // fixed order.  Each warp also sums v(c) times its partial products: the
            // block's part of y.v without a block reduction of its own.
            {
                double yvw = 0.0;
                for (int item = warp; item < nitems; item += NW) {
                    const int g = item % nq, rb = item / nq, m0 = mB + 4 * g;
                    const int R0 = rs + 512 * rb;
                    const double2* col[4];
#pragma unroll
                    for (int c = 0; c < 4; ++c)
                        col[c] = reinterpret_cast<const double2*>(A + (size_t)(rank + CL * min(m0 + c, cnt - 1)) * n + R0);
                    const double2* vp = reinterpret_cast<const double2*>(vv + R0 + par);
                    double sc[4] = {0.0, 0.0, 0.0, 0.0};
                    const int np = (n - R0) / 2;   // whole pairs from R0 on
                    constexpr int UB = 4;           // pairs per lane and column in one batch of loads
                    if (np >= 256) {
#pragma unroll
                        for (int h = 0; h < 8 / UB; ++h) {
                            double2 x[4][UB], xv[UB];
#pragma unroll
                            for (int u = 0; u < UB; ++u) {
                                const int pp = lane + 32 * (UB * h + u);
                                xv[u] = vp[pp];
#pragma unroll
                                for (int c = 0; c < 4; ++c) x[c][u] = col[c][pp];
                            }
#pragma unroll
                            for (int u = 0; u < UB; ++u)
#pragma unroll
                                for (int c = 0; c < 4; ++c) sc[c] = fma(x[c][u].y, xv[u].y, fma(x[c][u].x, xv[u].x, sc[c]));
                        }
                    } else {
                        // the last row batch: whole pairs, then a last single row when n - R0 is odd
                        for (int h = 0; h < 8 / UB; ++h) {
                            double2 x[4][UB], xv[UB];
#pragma unroll
                            for (int u = 0; u < UB; ++u) {
                                const int pp = lane + 32 * (UB * h + u);
                                const bool in = pp < np, one = pp == np && R0 + 2 * pp == n - 1;
                                const double* vs = vv + R0 + par + 2 * pp;
                                xv[u] = in ? vp[pp] : make_double2(one ? vs[0] : 0.0, 0.0);
#pragma unroll
                                for (int c = 0; c < 4; ++c) {
                                    const double* as = reinterpret_cast<const double*>(col[c] + pp);
                                    x[c][u] = in ? col[c][pp] : make_double2(one ? as[0] : 0.0, 0.0);
                                }
                            }
#pragma unroll
                            for (int u = 0; u < UB; ++u)
#pragma unroll
                                for (int c = 0; c < 4; ++c) sc[c] = fma(x[c][u].y, xv[u].y, fma(x[c][u].x, xv[u].x, sc[c]));
                        }
                    }
                    const double tot = warp_sum4(sc[0], sc[1], sc[2], sc[3], lane);
                    const int mc4 = m0 + ((lane >> 3) & 3);
                    if ((lane & 7) == 0 && mc4 < cnt) {
                        ysp[rb * MM + mc4] = tot;
                        yvw = fma(tot, vj[mc4], yvw);
                    }
                }
                yvw += __shfl_xor_sync(0xffffffffu, yvw, 8);
                yvw += __shfl_xor_sync(0xffffffffu, yvw, 16);
                if (lane == 0) red[warp] = yvw;
                __syncthreads();
            }
            const int mc = mB + tid;
            const bool own_c = mc < cnt;
            if (own_c) {
                double sy = 0.0;
                for (int rb = 0; rb < nrb; ++rb) sy += ysp[rb * MM + mc];
                ys[mc] = sy;
                if (tid == 0 && pivot_owner && k + 1 <= last)
                    for (int r = 0; r < CL; ++r) cluster.map_shared_rank(Y1, r)[0] = sy;
            }
            if (tid < CL) {
                double yvp = 0.0;
                for (int w = 0; w < NW; ++w) yvp += red[w];   // the same order in every block
                cluster.map_shared_rank(P2, tid)[rank * P2W + 2 * NB] = yvp;
            }
            cluster.sync();
            // ---- C: totals, w of the own rows and of the next pivot row ----
            if (tid < 2 * j) {
                const int o = tid < j ? tid : NB + (tid - j);
                double s = 0.0;
                for (int r = 0; r < CL; ++r) s += P2[r * P2W + o];
                tsum[o] = s;
            } else if (tid == TT - 1) {
                double s = 0.0;
                for (int r = 0; r < CL; ++r) s += P2[r * P2W + 2 * NB];
                tsum[2 * NB] = s;
            }
            __syncthreads();
            double t12 = 0.0, t12b = 0.0;
            #pragma unroll 4
            for (int q = 0; q + 1 < j; q += 2) {
                t12 = fma(tsum[q], tsum[NB + q], t12);
                t12b = fma(tsum[q + 1], tsum[NB + q + 1], t12b);
            }
            if (j & 1) t12 = fma(tsum[j - 1], tsum[NB + j - 1], t12);
            const double wv = tau * (tsum[2 * NB] - 2.0 * (t12 + t12b));
            const double al = -0.5 * tau * wv;
            if (own_c) WO[j * MM + mc] = w_entry(ys[mc], VO + mc, WO + mc, MM, tsum, tsum + NB, j, tau, al, vj[mc]);
            if (k + 1 <= last) {
                if (tid < j) {
                    piv[tid] = pivn[NB + tid];        // W(k+1, q)
                    piv[NB + tid] = pivn[tid];        // V(k+1, q)
                } else if (tid == TT - 1) {
                    piv[j] = w_entry(Y1[0], pivn, pivn + NB, 1, tsum, tsum + NB, j, tau, al, 1.0);
                    piv[NB + j] = 1.0;
                }
            }
            __syncthreads();
        }
        // ---- the panel's V, W, reflectors (into A below the subdiagonal), D, E and tau go
        // to global memory once per panel: a global store pending at a cluster barrier
        // makes the barrier wait for it ----
        const int m1 = first_own(p + 1), nm1 = cnt - m1;
        for (int e = tid; e < jn * nm1; e += TT) {
            const int mm = m1 + e % nm1, q = e / nm1;
            const int i = rank + CL * mm, kq = p + q;
            if (i >= kq + 1) {
                const double v = VO[q * MM + mm];
                Vg[(size_t)i + (size_t)q * n] = v;
                Wg[(size_t)i + (size_t)q * n] = WO[q * MM + mm];
                if (i > kq + 1) A[(size_t)i + (size_t)kq * n] = v;
            }
        }
        if (tid < jn) {
            const int kq = p + tid;
            if (kq % CL == rank) L.D[kq] = pan[tid];
            if (rank == 0) { L.E[kq] = pan[NB + tid]; L.TAU[kq] = pan[2 * NB + tid]; }
        }
        // ---- trailing update of the own columns l >= r0, rows >= r0 ----
        const int r0 = last + 1, jc = last - p + 1;
        cluster.sync();
        const int mR = first_own(r0);
        // register tiles of 4 rows (tr + 32 u) x 4 own columns (4 tc + c), K = 2 jc
        const int tr = tid & 31, tc = tid >> 5;
        for (int ib = r0; ib < n; ib += TRW) {
            for (int e = tid; e < jc * TRW; e += TT) {
                const int q = e / TRW, r = e % TRW, row = ib + r;
                stV[q * TRW + r] = row < n ? __ldcg(Vg + row + (size_t)q * n) : 0.0;
                stW[q * TRW + r] = row < n ? __ldcg(Wg + row + (size_t)q * n) : 0.0;
            }
            __syncthreads();
            for (int mc = mR; mc < cnt; mc += 4 * (TT / 32)) {
                const int m0 = mc + 4 * tc;
                if (m0 < cnt) {
                    int mcol[4];
#pragma unroll
                    for (int c = 0; c < 4; ++c) mcol[c] = min(m0 + c, cnt - 1);
                    double acc[4][4];
#pragma unroll
                    for (int u = 0; u < 4; ++u)
#pragma unroll
                        for (int c = 0; c < 4; ++c) acc[u][c] = 0.0;
                    for (int q = 0; q < jc; ++q) {
                        double av[4], aw[4], bw[4], bv[4];
#pragma unroll
                        for (int u = 0; u < 4; ++u) {
                            av[u] = stV[q * TRW + tr + 32 * u];
                            aw[u] = stW[q * TRW + tr + 32 * u];
                        }
#pragma unroll
                        for (int c = 0; c < 4; ++c) {
                            bw[c] = WO[q * MM + mcol[c]];
                            bv[c] = VO[q * MM + mcol[c]];
                        }
#pragma unroll
                        for (int u = 0; u < 4; ++u)
#pragma unroll
                            for (int c = 0; c < 4; ++c) acc[u][c] = fma(av[u], bw[c], fma(aw[u], bv[c], acc[u][c]));
                    }
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        if (m0 + c >= cnt) continue;
                        double* colp = A + (size_t)(rank + CL * (m0 + c)) * n;
#pragma unroll
                        for (int u = 0; u < 4; ++u) {
                            const int row = ib + tr + 32 * u;
                            if (row < n) colp[row] -= acc[u][c];
                        }
                    }
                }
            }
            __syncthreads();
        }
    }
    if ((n - 1) % CL == rank && tid == 0) L.D[n - 1] = A[(size_t)(n - 1) + (size_t)(n - 1) * n];
    if (rank == 0 && tid == 0) L.E[n - 1] = 0.0;
    cluster.sync();   // no block leaves while another may still write its shared memory
}

// ---------------------------------------------------------------------------------
// the same cluster tridiagonalisation on the lower triangle only
// ---------------------------------------------------------------------------------
// k_tri_cluster streams every own column of the trailing matrix in full for each column
// step's product y = A v, and updates full columns after each panel.  The matrix is
// symmetric, so this variant keeps and reads only the lower triangle: the product of own
// column l takes rows i >= l,
//   y(l) += sum_{i >= l} A(i, l) v(i)        (the column's own dot product)
//   z(i) += A(i, l) v(l)       for i > l     (row i's share of A(i, :) v, i.e. the upper
//                                             triangle read as the transpose)
// and every block sends the z of each row to the block that owns the row, in the same
// cluster exchange that carries the panel dot products; y(l) = dot(l) + the received z.
// Half the bytes of the product and of the panel update cross from L2.
// Work split of the product: the trailing rows form blocks of 32; each warp takes whole
// row blocks (dealt heaviest first, in snake order, so the warps' loads balance), one row
// per lane, and walks the own columns that reach the block in tiles of 32: the loads are
// coalesced along the rows, z of the lane's row stays in a register across the tiles, and
// the 32 column dot products of a tile are summed over the lanes by a transposed
// butterfly (31 shuffles; lane j ends with column j).  Each warp adds its column partials
// into its own row of ysp, and the warps' partials are added in warp order, so results do
// not depend on the schedule.
// The panel rows of column p+q (needed as own rows of the column) are read from the column
// itself (rows at stride CL), since the upper triangle is stale.
struct TriLayoutS {
    int MM, PN;   // own indices per block, rows (even)
    __host__ __device__ long long doubles(int CL) const {
        const long long stage = (long long)NB * MM > 2LL * NB * TRW ? (long long)NB * MM : 2LL * NB * TRW;
        return 2LL * NB * MM + PN + MM + (long long)CL * P2W + CL + 2 + 2LL * NB + 2LL * NB + P2W + 32 +
               stage + (long long)(TT / 32) * MM + (long long)CL * MM + 3LL * NB;
    }
};

// v[0..31] of every lane summed over the warp: lane j returns the sum of v[j]
__device__ __forceinline__ double transpose_sum32(double (&v)[32], int lane) {
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
        const bool upper = (lane & o) != 0;
#pragma unroll
        for (int i = 0; i < o; ++i) {
            const double send = upper ? v[i] : v[i + o];
            const double keep = upper ? v[i + o] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
    }
    return v[0];
}

template <int CL>
__global__ void __launch_bounds__(TT, 1) k_tri_csym(const LSec* __restrict__ secs, TriLayoutS lay,
                                                   double* eigbuf, double* wsd, int* wsi) {
    extern __shared__ double sm[];
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    const LSec sec = secs[blockIdx.x / CL];
    LView L = lview(sec, eigbuf, wsd, wsi);
    const int n = L.n, MM = lay.MM, PN = lay.PN;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = TT / 32;
    double* VO = sm;                       // NB x MM: V(own row m, q) at q*MM + m
    double* WO = VO + (size_t)NB * MM;     // NB x MM
    double* cv = WO + (size_t)NB * MM;     // column k (rows > k), then v, by row
    double* ys = cv + PN;                  // y of the own columns
    double* P2 = ys + MM;                  // CL x P2W partials, by source block
    double* redA = P2 + CL * P2W;          // CL partial |x|^2
    double* Y1 = redA + CL;                // y(k+1) from its owner
    double* pivn = Y1 + 2;                 // 2 NB: V(k+1, q) | W(k+1, q) from its owner
    double* piv = pivn + 2 * NB;           // 2 NB: W(k, q) | V(k, q) of the current pivot row
    double* tsum = piv + 2 * NB;           // t1 | t2 | y.v
    double* red = tsum + P2W;              // 32
    double* AR = red + 32;                 // NB x MM: A(own row m, p + q), during the columns
    double* stV = AR;                      // NB x TRW staged rows of V (transposed), panel update
    double* stW = stV + NB * TRW;          // NB x TRW
    double* ysp = AR + ((size_t)NB * MM > 2 * NB * TRW ? (size_t)NB * MM : 2 * NB * TRW);   // NW x MM
    double* zr = ysp + (size_t)NW * MM;         // CL x MM: z of the own rows, by source block
    double* pan = zr + (size_t)CL * MM;         // D | E | tau of the panel's columns
    double* Vg = L.VW;
    double* Wg = L.VW + (size_t)NB * n;
    double* A = L.A;
    const int cnt = (n - rank + CL - 1) / CL;                           // own indices rank + CL*m
    auto first_own = [&](int i0) { return (i0 - rank + CL - 1) / CL; };  // i0 >= 0
    (void)PN;

    for (int p = 0; p < n - 1; p += NB) {
        const int last = min(p + NB - 1, n - 2);
        const int jn = last - p + 1;
        // own rows i >= p + q of the panel's columns p + q (lower triangle, stride CL)
        {
            const int m0 = first_own(p);
            const int nm = cnt - m0;
            for (int e = tid; e < jn * nm; e += TT) {
                const int q = e / nm, m = m0 + e % nm, i = rank + CL * m;
                if (i >= p + q) AR[q * MM + m] = __ldcg(A + (size_t)i + (size_t)(p + q) * n);
            }
        }
        __syncthreads();
        for (int k = p; k <= last; ++k) {
            const int j = k - p;
            // ---- A: own rows of column k, broadcast ----
            const int m = first_own(k) + tid;
            const bool act = m < cnt;
            const int i = rank + CL * m;
            double c = 0.0, ss = 0.0;
            if (act) {
                double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
                int q = 0;
                for (; q + 1 < j; q += 2) {
                    s0 = fma(VO[q * MM + m], piv[q], s0);
                    s1 = fma(WO[q * MM + m], piv[NB + q], s1);
                    s2 = fma(VO[(q + 1) * MM + m], piv[q + 1], s2);
                    s3 = fma(WO[(q + 1) * MM + m], piv[NB + q + 1], s3);
                }
                if (q < j) {
                    s0 = fma(VO[q * MM + m], piv[q], s0);
                    s1 = fma(WO[q * MM + m], piv[NB + q], s1);
                }
                c = AR[j * MM + m] - ((s0 + s2) + (s1 + s3));
                if (i == k) pan[j] = c;
                if (i >= k + 2) ss = c * c;
                if (i >= k + 1)
                    for (int r = 0; r < CL; ++r) cluster.map_shared_rank(cv, r)[i] = c;
            }
            const double ssb = block_sum(ss, red);
            if (tid < CL) cluster.map_shared_rank(redA, tid)[rank] = ssb;
            cluster.sync();
            double xn2 = 0.0;
            for (int r = 0; r < CL; ++r) xn2 += redA[r];
            const double alpha = cv[k + 1];
            double beta = alpha, tau = 0.0, scal = 0.0;
            if (xn2 != 0.0) {
                beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
                tau = (beta - alpha) / beta;
                scal = 1.0 / (alpha - beta);
            }
            for (int r = k + 2 + tid; r < n; r += TT) cv[r] = xn2 == 0.0 ? 0.0 : cv[r] * scal;
            if (act && i >= k + 1) VO[j * MM + m] = (i == k + 1) ? 1.0 : (xn2 == 0.0 ? 0.0 : c * scal);
            if (tid == 0) { pan[NB + j] = beta; pan[2 * NB + j] = tau; }
            const int mB = first_own(k + 1);
            for (int mm = mB + lane; mm < cnt; mm += 32) ysp[warp * MM + mm] = 0.0;
            __syncthreads();
            // ---- B: partial W^T v, V^T v over the own rows, the next pivot row, the
            // lower-triangle product, z to the row owners, partial y.v ----
            const double* vj = VO + j * MM;
            for (int o = warp; o < 2 * j; o += NW) {
                const double* colp = (o < j) ? WO + o * MM : VO + (o - j) * MM;
                double s = 0.0;
                for (int mm = mB + lane; mm < cnt; mm += 32) s = fma(colp[mm], vj[mm], s);
                s = warp_sum(s);
                if (lane < CL) cluster.map_shared_rank(P2, lane)[rank * P2W + (o < j ? o : NB + (o - j))] = s;
            }
            const bool pivot_owner = (rank == (k + 1) % CL);
            if (pivot_owner && k + 1 <= last) {
                for (int e = tid; e < 2 * j * CL; e += TT) {
                    const int q = e / CL, r = e % CL;
                    const double val = q < j ? VO[q * MM + mB] : WO[(q - j) * MM + mB];
                    cluster.map_shared_rank(pivn, r)[q < j ? q : NB + (q - j)] = val;
                }
            }
            double yvp = 0.0;   // this block's part of v^T A v
            {
                const int nblk = (n - k - 1 + 31) / 32;
                double* yw = ysp + (size_t)warp * MM;
                for (int pass = 0; pass * NW < nblk; ++pass) {
                    const int slot = (pass & 1) ? NW - 1 - warp : warp;
                    const int qi = pass * NW + slot;
                    if (qi >= nblk) continue;
                    const int b = nblk - 1 - qi;            // heaviest (lowest) blocks first
                    const int r0b = k + 1 + 32 * b;
                    const int r = r0b + lane;
                    const double vr = r < n ? (r == k + 1 ? 1.0 : cv[r]) : 0.0;   // v(k+1) = 1
                    const int lastrow = min(r0b + 31, n - 1);
                    const int mLim = min(cnt, (lastrow - rank) / CL + 1);   // own columns l <= lastrow
                    double z = 0.0;
                    for (int t0 = mB; t0 < mLim; t0 += 32) {
                        double d[32];
#pragma unroll
                        for (int jj = 0; jj < 32; ++jj) {
                            const int mc = t0 + jj;
                            const int l = rank + CL * mc;
                            d[jj] = (mc < mLim && r < n && r >= l) ? A[(size_t)l * n + r] : 0.0;
                        }
#pragma unroll
                        for (int jj = 0; jj < 32; ++jj) {
                            const int mc = t0 + jj;
                            const int l = rank + CL * mc;
                            const double x = d[jj];
                            if (mc < mLim && r > l) z = fma(x, l == k + 1 ? 1.0 : cv[l], z);
                            d[jj] = x * vr;
                        }
                        const double dsum = transpose_sum32(d, lane);
                        if (t0 + lane < mLim) yw[t0 + lane] += dsum;
                    }
                    if (r < n) {
                        cluster.map_shared_rank(zr, r % CL)[rank * MM + r / CL] = z;
                        yvp = fma(vr, z, yvp);
                    }
                }
            }
            __syncthreads();
            const int mc = mB + tid;
            const bool own_c = mc < cnt;
            if (own_c) {
                double dot = 0.0;
                for (int w = 0; w < NW; ++w) dot += ysp[w * MM + mc];
                ys[mc] = dot;
                yvp = fma(vj[mc], dot, yvp);
                // y(k+1) has no z part (no own column lies left of it in the trailing block)
                if (pivot_owner && k + 1 <= last && rank + CL * mc == k + 1)
                    for (int r = 0; r < CL; ++r) cluster.map_shared_rank(Y1, r)[0] = dot;
            }
            yvp = block_sum(yvp, red);
            if (tid < CL) cluster.map_shared_rank(P2, tid)[rank * P2W + 2 * NB] = yvp;
            cluster.sync();
            // ---- C: totals, y of the own columns, w of the own rows and of the next pivot row ----
            if (own_c) {
                double zz = 0.0;
                for (int r = 0; r < CL; ++r) zz += zr[r * MM + mc];
                ys[mc] += zz;
            }
            if (tid < 2 * j) {
                const int o = tid < j ? tid : NB + (tid - j);
                double s = 0.0;
                for (int r = 0; r < CL; ++r) s += P2[r * P2W + o];
                tsum[o] = s;
            } else if (tid == TT - 1) {
                double s = 0.0;
                for (int r = 0; r < CL; ++r) s += P2[r * P2W + 2 * NB];
                tsum[2 * NB] = s;
            }
            __syncthreads();
            double t12 = 0.0, t12b = 0.0;
            for (int q = 0; q + 1 < j; q += 2) {
                t12 = fma(tsum[q], tsum[NB + q], t12);
                t12b = fma(tsum[q + 1], tsum[NB + q + 1], t12b);
            }
            if (j & 1) t12 = fma(tsum[j - 1], tsum[NB + j - 1], t12);
            const double wv = tau * (tsum[2 * NB] - 2.0 * (t12 + t12b));
            const double al = -0.5 * tau * wv;
            if (own_c) WO[j * MM + mc] = w_entry(ys[mc], VO + mc, WO + mc, MM, tsum, tsum + NB, j, tau, al, vj[mc]);
            if (k + 1 <= last) {
                if (tid < j) {
                    piv[tid] = pivn[NB + tid];        // W(k+1, q)
                    piv[NB + tid] = pivn[tid];        // V(k+1, q)
                } else if (tid == TT - 1) {
                    piv[j] = w_entry(Y1[0], pivn, pivn + NB, 1, tsum, tsum + NB, j, tau, al, 1.0);
                    piv[NB + j] = 1.0;
                }
            }
            __syncthreads();
        }
        // ---- the panel's V, W, reflectors, D, E, tau to global memory ----
        const int m1 = first_own(p + 1), nm1 = cnt - m1;
        for (int e = tid; e < jn * nm1; e += TT) {
            const int mm = m1 + e % nm1, q = e / nm1;
            const int i = rank + CL * mm, kq = p + q;
            if (i >= kq + 1) {
                const double v = VO[q * MM + mm];
                Vg[(size_t)i + (size_t)q * n] = v;
                Wg[(size_t)i + (size_t)q * n] = WO[q * MM + mm];
                if (i > kq + 1) A[(size_t)i + (size_t)kq * n] = v;
            }
        }
        if (tid < jn) {
            const int kq = p + tid;
            if (kq % CL == rank) L.D[kq] = pan[tid];
            if (rank == 0) { L.E[kq] = pan[NB + tid]; L.TAU[kq] = pan[2 * NB + tid]; }
        }
        // ---- lower-triangle update of the own columns l >= r0: rows >= l ----
        const int r0 = last + 1, jc = last - p + 1;
        cluster.sync();
        const int mR = first_own(r0);
        const int tr = tid & 31, tc = tid >> 5;
        for (int ib = r0; ib < n; ib += TRW) {
            // own columns that reach this chunk: rank + CL*m <= its last row
            const int lastrow = min(ib + TRW, n) - 1;
            const int mLim = lastrow >= rank ? min(cnt, (lastrow - rank) / CL + 1) : 0;
            if (mLim <= mR) continue;   // no own column reaches this chunk yet (uniform in the block)
            for (int e = tid; e < jc * TRW; e += TT) {
                const int q = e / TRW, rr = e % TRW, row = ib + rr;
                stV[q * TRW + rr] = row < n ? __ldcg(Vg + row + (size_t)q * n) : 0.0;
                stW[q * TRW + rr] = row < n ? __ldcg(Wg + row + (size_t)q * n) : 0.0;
            }
            __syncthreads();
            for (int mc2 = mR; mc2 < mLim; mc2 += 4 * (TT / 32)) {
                const int m0 = mc2 + 4 * tc;
                if (m0 < mLim) {
                    int mcol[4];
#pragma unroll
                    for (int cc = 0; cc < 4; ++cc) mcol[cc] = min(m0 + cc, mLim - 1);
                    double acc[4][4];
#pragma unroll
                    for (int u = 0; u < 4; ++u)
#pragma unroll
                        for (int cc = 0; cc < 4; ++cc) acc[u][cc] = 0.0;
                    for (int q = 0; q < jc; ++q) {
                        double av[4], aw[4], bw[4], bv[4];
#pragma unroll
                        for (int u = 0; u < 4; ++u) {
                            av[u] = stV[q * TRW + tr + 32 * u];
                            aw[u] = stW[q * TRW + tr + 32 * u];
                        }
#pragma unroll
                        for (int cc = 0; cc < 4; ++cc) {
                            bw[cc] = WO[q * MM + mcol[cc]];
                            bv[cc] = VO[q * MM + mcol[cc]];
                        }
#pragma unroll
                        for (int u = 0; u < 4; ++u)
#pragma unroll
                            for (int cc = 0; cc < 4; ++cc)
                                acc[u][cc] = fma(av[u], bw[cc], fma(aw[u], bv[cc], acc[u][cc]));
                    }
#pragma unroll
                    for (int cc = 0; cc < 4; ++cc) {
                        if (m0 + cc >= mLim) continue;
                        const int l = rank + CL * (m0 + cc);
                        double* colp = A + (size_t)l * n;
#pragma unroll
                        for (int u = 0; u < 4; ++u) {
                            const int row = ib + tr + 32 * u;
                            if (row < n && row >= l) colp[row] -= acc[u][cc];
                        }
                    }
                }
            }
            __syncthreads();
        }
        // the next panel reads its columns' own rows from columns that other blocks own
        // and have just updated: their stores are visible after this barrier
        cluster.sync();
    }
    if ((n - 1) % CL == rank && tid == 0) L.D[n - 1] = A[(size_t)(n - 1) + (size_t)(n - 1) * n];
    if (rank == 0 && tid == 0) L.E[n - 1] = 0.0;
    cluster.sync();   // no block leaves while another may still write its shared memory
}

__global__ void k_tri_end(const LSec* __restrict__ secs, double* eigbuf, double* wsd, int* wsi) {
    const LSec sec = secs[blockIdx.x];
    if (threadIdx.x != 0) return;
    LView L = lview(sec, eigbuf, wsd, wsi);
    const int n = L.n;
    L.D[n - 1] = L.A[(size_t)(n - 1) + (size_t)(n - 1) * n];
    L.E[n - 1] = 0.0;
}

// ---------------------------------------------------------------------------------
// divide and conquer
// ---------------------------------------------------------------------------------
// leaves of the divide and conquer: one block per aligned range of DC_LOW rows of a
// sector runs every merge inside that range (all merges up to DC_LOW rows stay inside)
__global__ void __launch_bounds__(512) k_dc_low(const LSec* __restrict__ secs, int nsec, double* eigbuf,
                                                double* wsd, int* wsi, int* status) {
    extern __shared__ double sm[];
    int bid = blockIdx.x, sidx = 0;
    for (; sidx < nsec; ++sidx) {
        const int nc = (secs[sidx].n + DC_LOW - 1) / DC_LOW;
        if (bid < nc) break;
        bid -= nc;
    }
    if (sidx >= nsec) return;
    LView L = lview(secs[sidx], eigbuf, wsd, wsi);
    const int n = L.n, tid = threadIdx.x, T = blockDim.x;
    const int c0 = bid * DC_LOW, c1 = min(c0 + DC_LOW, n), nl = c1 - c0;
    double* red = sm;
    double* gsm = sm + 32;
    // D of the range and the merge vectors in shared memory; the merges work in indices
    // local to the range (Z, U, Qt through pointers to the range's diagonal block)
    double* Dl = gsm + nrg::kCtaGemmSmem;
    const Scratch Sl = scratch_smem(Dl, DC_LOW);
    double* Zl = L.Z + c0 + (size_t)c0 * n;
    double* Ul = L.U + c0 + (size_t)c0 * n;
    double* Ql = L.Qt + c0 + (size_t)c0 * n;
    const double* El = L.E + c0;
    // columns c0 .. c1-1 of Z start as the identity
    const long long ne = (long long)n * (c1 - c0);
    for (long long e = tid; e < ne; e += T) {
        const long long col = c0 + e / n, row = e % n;
        L.Z[row + col * n] = (row == col) ? 1.0 : 0.0;
    }
    // rank-one tearing at every boundary: each leaf is 1 x 1
    for (int i = c0 + tid; i < c1; i += T) {
        double dv = L.D[i];
        if (i > 0) dv -= fabs(L.E[i - 1]);
        if (i < n - 1) dv -= fabs(L.E[i]);
        Dl[i - c0] = dv;
    }
    __syncthreads();
    const int warp = tid >> 5, lane = tid & 31, nwarps = T >> 5;
    for (int s = 1; 2 * s <= DC_LOW && s < nl; s *= 2) {
        if (2 * s <= 32) {
            WarpG wg{lane};
            int mi = 0;
            for (int a = 0; a + s < nl; a += 2 * s, ++mi) {
                if (mi % nwarps != warp) continue;
                dc_merge(wg, a, a + s, min(a + 2 * s, nl), n, Zl, Dl, El, Sl, Ul, Ql, red, gsm, status);
            }
            __syncthreads();
        } else {
            BlockG bg;
            for (int a = 0; a + s < nl; a += 2 * s)
                dc_merge(bg, a, a + s, min(a + 2 * s, nl), n, Zl, Dl, El, Sl, Ul, Ql, red, gsm, status);
        }
    }
    __syncthreads();
    for (int i = tid; i < nl; i += T) L.D[c0 + i] = Dl[i];
}

struct Merge {
    int sec, a, mid, b;
    // block ranges of the parallel phases for the three thread mappings: one thread per
    // item (kMapItem), one warp per item (kMapWarp), one thread per few matrix entries
    // of the nn x nn merged block (kMapWide)
    int blk0[3], nblk[3];
};
constexpr int kMapItem = 0, kMapWarp = 1, kMapWide = 2;
constexpr int kWideItems = 8;   // matrix entries per thread in kMapWide

__device__ int find_merge(const Merge* ms, int nm, int map) {
    int lo = 0, hi = nm - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (ms[mid].blk0[map] <= (int)blockIdx.x) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__global__ void __launch_bounds__(512) k_dc_prep(const LSec* __restrict__ secs, const Merge* __restrict__ ms,
                                                 double* eigbuf, double* wsd, int* wsi) {
    __shared__ double red[32];
    const Merge m = ms[blockIdx.x];
    LView L = lview(secs[m.sec], eigbuf, wsd, wsi);
    merge_prep(BlockG{}, m.a, m.mid, m.b, L.n, L.Z, L.D, L.E, L.S, red);
}

// phase 1 roots, 2 zhat, 3 rank-one vectors + values (one warp per root / entry / column),
// 4 final order + GEMM index lists (one thread per item), 5 deflated copies, 6 copy back
// (one thread per few entries)
__global__ void __launch_bounds__(TPB) k_dc_phase(const LSec* __restrict__ secs, const Merge* __restrict__ ms,
                                                  int nm, int phase, double* eigbuf, double* wsd, int* wsi,
                                                  int* status) {
    const int map = phase <= 3 ? kMapWarp : (phase == 4 ? kMapItem : kMapWide);
    const int mi = find_merge(ms, nm, map);
    const Merge m = ms[mi];
    LView L = lview(secs[m.sec], eigbuf, wsd, wsi);
    const int t = ((int)blockIdx.x - m.blk0[map]) * blockDim.x + threadIdx.x;
    const int T = m.nblk[map] * blockDim.x;
    const WarpLanes wl{(int)(threadIdx.x & 31)};
    switch (phase) {
        case 1: merge_roots(t >> 5, T >> 5, m.a, m.mid, L.E, L.S, status, wl); break;
        case 2: merge_zhat(t >> 5, T >> 5, m.a, m.mid, L.E, L.S, wl); break;
        case 3:
            merge_ucols(t >> 5, T >> 5, m.a, L.n, L.S, L.U, wl);
            merge_vals(t, T, m.a, m.b, L.S);
            break;
        case 4: {
            merge_rank(t, T, m.a, m.b, L.S);
            const int K = L.S.mk[m.a];
            // gathered columns of Z for the GEMM: a + perm[nd[q]] (ra reused after prep)
            for (int q = t; q < K; q += T) L.S.ra[m.a + q] = m.a + L.S.perm[m.a + L.S.nd[m.a + q]];
            break;
        }
        case 5: merge_deflated(t, T, m.a, m.b, L.n, L.Z, L.Qt, L.S); break;
        case 6: merge_copyback(t, T, m.a, m.b, L.n, L.Z, L.D, L.Qt, L.S); break;
        default: break;
    }
}

// scatter columns a + pos[j] of the nondeflated eigenvectors (rb reused)
__global__ void k_dc_poscols(const LSec* __restrict__ secs, const Merge* __restrict__ ms, int nm,
                             double* eigbuf, double* wsd, int* wsi) {
    const int mi = find_merge(ms, nm, kMapItem);
    const Merge m = ms[mi];
    LView L = lview(secs[m.sec], eigbuf, wsd, wsi);
    const int t = ((int)blockIdx.x - m.blk0[kMapItem]) * blockDim.x + threadIdx.x;
    const int T = m.nblk[kMapItem] * blockDim.x;
    const int K = L.S.mk[m.a];
    for (int j = t; j < K; j += T) L.S.rb[m.a + j] = m.a + L.S.pos[m.a + j];
}

// ---------------------------------------------------------------------------------
// back-transformation
// ---------------------------------------------------------------------------------
// explicit V panel (mr x b, ld mr) of reflectors jb .. jb+b-1 into U
__global__ void k_bt_vpanel(const LSec* __restrict__ secs, int q, double* eigbuf, double* wsd, int* wsi) {
    const LSec sec = secs[blockIdx.y];
    const int n = sec.n, nr = n - 1, jb = q * NBB;
    if (jb >= nr) return;
    LView L = lview(sec, eigbuf, wsd, wsi);
    const int b = min(NBB, nr - jb), r0 = jb + 1, mr = n - r0;
    const long long tot = (long long)mr * b;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot; e += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(e % mr), c = (int)(e / mr);
        const int k = jb + c, row = r0 + i;
        double v = 0.0;
        if (row == k + 1) v = 1.0;
        else if (row > k + 1) v = L.A[(size_t)row + (size_t)k * n];
        L.U[e] = v;
    }
}

// triangular factor T of the panel from the Gram matrix G (in Qt, b x b) and tau; T goes
// to Qt + NBB*NBB (b x b, ld NBB)
__global__ void k_bt_tfactor(const LSec* __restrict__ secs, int q, double* eigbuf, double* wsd, int* wsi) {
    extern __shared__ double tsm[];
    double* Ts = tsm;               // NBB x NBB
    double* G = tsm + NBB * NBB;    // the Gram matrix, staged
    const LSec sec = secs[blockIdx.x];
    const int n = sec.n, nr = n - 1, jb = q * NBB;
    if (jb >= nr) return;
    LView L = lview(sec, eigbuf, wsd, wsi);
    const int b = min(NBB, nr - jb);
    const int p = threadIdx.x;
    for (int e = threadIdx.x; e < NBB * NBB; e += blockDim.x) {
        Ts[e] = 0.0;
        G[e] = L.Qt[e];
    }
    __syncthreads();
    for (int c = 0; c < b; ++c) {
        const double tc = L.TAU[jb + c];
        double acc = 0.0;
        if (p < c)
            for (int qq = p; qq < c; ++qq) acc += Ts[p + qq * NBB] * (-tc * G[qq + c * NBB]);
        __syncthreads();
        if (p < c) Ts[p + c * NBB] = acc;
        if (p == 0) Ts[c + c * NBB] = tc;
        __syncthreads();
    }
    for (int e = threadIdx.x; e < NBB * NBB; e += blockDim.x) L.Qt[NBB * NBB + e] = Ts[e];
}

// ---- back-transformation in one pass per column block --------------------------------
// Panel q holds reflectors jb = 64 q .. jb + b - 1 (rows r0 = jb + 1 .. n - 1).  In R:
// the triangular factors T_q (NBB x NBB each) first, then the explicit panels
// V_q (mr x NBB, column-major, zero beyond b).
__device__ __forceinline__ long long bt_panel_off(int n, int q) {
    const long long npan = (n - 2) / NBB + 1;
    const long long before = (long long)q * (n - 1) - (long long)NBB * q * (q - 1) / 2;   // sum of mr
    return npan * NBB * NBB + (long long)NBB * before;
}

// explicit V_q, its Gram matrix and T_q (dlarft, forward, columnwise) for every panel of
// every sector at once: one block per (panel, sector)
__global__ void __launch_bounds__(256) k_bt_prep(const LSec* __restrict__ secs, double* eigbuf, double* wsd,
                                                 int* wsi) {
    extern __shared__ double bsm[];
    double* Vs = bsm;                  // chunk of the panel, Vs[c * 65 + r]
    double* G = Vs + NBB * 65;         // NBB x NBB, column-major
    double* Ts = G + NBB * NBB;        // NBB x NBB, column-major
    const LSec sec = secs[blockIdx.y];
    const int n = sec.n, nr = n - 1, q = blockIdx.x, jb = q * NBB;
    if (jb >= nr) return;
    LView L = lview(sec, eigbuf, wsd, wsi);
    const int b = min(NBB, nr - jb), r0 = jb + 1, mr = n - r0;
    double* Rp = L.R + bt_panel_off(n, q);
    double* Tq = L.R + (size_t)q * NBB * NBB;
    const int tid = threadIdx.x, ti = tid & 15, tj = tid >> 4;
    double g[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int c = 0; c < 4; ++c) g[a][c] = 0.0;
    for (int i0 = 0; i0 < mr; i0 += 64) {
        const int rows = min(64, mr - i0);
        for (int e = tid; e < 64 * NBB; e += 256) {
            const int r = e & 63, c = e >> 6;
            const int row = r0 + i0 + r, k = jb + c;
            double v = 0.0;
            if (r < rows && c < b) v = (row == k + 1) ? 1.0 : (row > k + 1 ? L.A[(size_t)row + (size_t)k * n] : 0.0);
            Vs[c * 65 + r] = v;
            if (r < rows) Rp[(size_t)(i0 + r) + (size_t)c * mr] = v;
        }
        __syncthreads();
        for (int r = 0; r < rows; ++r) {
            double x[4], y[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                x[a] = Vs[(ti * 4 + a) * 65 + r];
                y[a] = Vs[(tj * 4 + a) * 65 + r];
            }
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int c = 0; c < 4; ++c) g[a][c] = fma(x[a], y[c], g[a][c]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int c = 0; c < 4; ++c) G[(ti * 4 + a) + (tj * 4 + c) * NBB] = g[a][c];
    for (int e = tid; e < NBB * NBB; e += 256) Ts[e] = 0.0;
    __syncthreads();
    for (int c = 0; c < b; ++c) {
        const double tc = L.TAU[jb + c];
        double acc = 0.0;
        if (tid < c)
            for (int qq = tid; qq < c; ++qq) acc += Ts[tid + qq * NBB] * (-tc * G[qq + c * NBB]);
        __syncthreads();
        if (tid < c) Ts[tid + c * NBB] = acc;
        if (tid == 0) Ts[c + c * NBB] = tc;
        __syncthreads();
    }
    for (int e = tid; e < NBB * NBB; e += 256) Tq[e] = Ts[e];
}

// 8-byte asynchronous global-to-shared copies (zero-filled when bytes is 0)
__device__ __forceinline__ void cp_async8(double* dst, const double* src, int bytes) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Z(:, c0 .. c0+CBK-1) <- H_0 ... H_{n-2} Z(:, ...) panel by panel (last panel first), the
// column block resident in shared memory; the result goes to the output
template <int CBK>
__global__ void __launch_bounds__(256, 1) k_bt_apply(const LSec* __restrict__ secs, int nsec, double* eigbuf,
                                                     double* wsd, int* wsi) {
    // The three small products of each panel, W = V^T Z, W2 = T W and Z -= V W2, on the
    // FP64 tensor pipe (mma.sync m8n8k4): the eight warps split the panel's 64 reflectors
    // (W, W2) or the chunk's 64 rows (the update) in slices of 8, and each warp covers the
    // CBK columns in tiles of 8.  What the products read streams through two shared
    // buffers of 64 x 65 doubles with asynchronous copies one step ahead: per panel the
    // chunks of 64 rows of V for W, then T, then the chunks again for the update, then the
    // next panel's first chunk.
    constexpr int NTJ = CBK / 8;
    // leading dimensions 4 mod 16 doubles (the Z block, the staged chunks and T): the
    // fragment loads and the row updates of a warp then fall on distinct bank pairs
    constexpr int VLD = NBB + 4;
    constexpr int BUF = NBB * VLD;
    extern __shared__ double asm_[];
    int bid = blockIdx.x, s = 0;
    for (; s < nsec; ++s) {
        const int nbk = (secs[s].n + CBK - 1) / CBK;
        if (bid < nbk) break;
        bid -= nbk;
    }
    if (s >= nsec) return;
    const LSec sec = secs[s];
    LView L = lview(sec, eigbuf, wsd, wsi);
    const int n = L.n, c0 = bid * CBK, nc = min(CBK, n - c0);
    const int ldz = n + ((4 - n) & 15);
    double* Zs = asm_;                      // Zs[j * ldz + row]
    double* Vb = Zs + (size_t)ldz * CBK;    // two buffers: Vs[c * VLD + r] (a chunk) or T (ld VLD)
    double* Ws = Vb + 2 * BUF;              // Ws[c * CBK + j]
    double* W2 = Ws + NBB * CBK;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, q4 = lane & 3;
    const int wr = 8 * warp;                // this warp's slice of reflectors / rows
    for (int j = 0; j < CBK; ++j)
        for (int row = tid; row < n; row += 256)
            Zs[(size_t)j * ldz + row] = j < nc ? L.Z[(size_t)row + (size_t)(c0 + j) * n] : 0.0;
    const int qmax = (n - 2) / NBB;
    // the load sequence: step t of panel q is a V chunk (t < C: for W; t > C: for the
    // update, chunk t - C - 1) or T (t == C), with C = ceil(mr / 64) chunks per pass
    auto chunks = [&](int q) { return (n - 1 - q * NBB + 63) / 64; };
    auto issue = [&](int q, int t, double* dst) {
        const int mr = n - 1 - q * NBB, C = chunks(q);
        if (t == C) {
            const double* Tq = L.R + (size_t)q * NBB * NBB;
            for (int e = tid; e < NBB * NBB; e += 256) cp_async8(dst + (e % NBB) + (e / NBB) * VLD, Tq + e, 8);
        } else {
            const int i0 = 64 * (t < C ? t : t - C - 1), rows = min(64, mr - i0);
            const double* Rp = L.R + bt_panel_off(n, q);
            for (int e = tid; e < 64 * NBB; e += 256) {
                const int r = e & 63, c = e >> 6;
                const int rr = r < rows ? r : rows - 1;   // in bounds; nothing is read when zero-filled
                cp_async8(dst + c * VLD + r, Rp + (size_t)(i0 + rr) + (size_t)c * mr, r < rows ? 8 : 0);
            }
        }
        cp_async_commit();
    };
    int buf = 0;
    issue(qmax, 0, Vb);
    for (int q = qmax; q >= 0; --q) {
        const int jb = q * NBB, r0 = jb + 1, mr = n - r0, C = chunks(q);
        double acc[NTJ][2];
#pragma unroll
        for (int t = 0; t < NTJ; ++t) acc[t][0] = acc[t][1] = 0.0;
        for (int t = 0; t <= 2 * C; ++t) {
            // the next step's load (the next panel's first chunk after the last step) into
            // the buffer the previous step has finished with
            double* nxt = Vb + (buf ^ 1) * BUF;
            if (t < 2 * C) issue(q, t + 1, nxt);
            else if (q > 0) issue(q - 1, 0, nxt);
            if (t < 2 * C || q > 0) cp_async_wait<1>();
            else cp_async_wait<0>();
            __syncthreads();
            const double* Vs = Vb + buf * BUF;
            if (t < C) {
                // W = V^T Z(r0:, :): W(i, j) for the warp's reflectors i
                const int i0 = 64 * t, rows = min(64, mr - i0);
                const double* zr = Zs + r0 + i0;
#pragma unroll 4
                for (int k0 = 0; k0 < 64; k0 += 4) {
                    const int kk = k0 + q4;
                    const double a = Vs[(wr + g) * VLD + kk];
#pragma unroll
                    for (int u = 0; u < NTJ; ++u) {
                        const double b = kk < rows ? zr[(size_t)(u * 8 + g) * ldz + kk] : 0.0;
                        nrg::cta_dmma(acc[u][0], acc[u][1], a, b);
                    }
                }
                if (t == C - 1) {
#pragma unroll
                    for (int u = 0; u < NTJ; ++u) {
                        Ws[(wr + g) * CBK + u * 8 + 2 * q4] = acc[u][0];
                        Ws[(wr + g) * CBK + u * 8 + 2 * q4 + 1] = acc[u][1];
                    }
                }
            } else if (t == C) {
                // W2 = T W (T upper triangular, zero below the diagonal)
#pragma unroll
                for (int u = 0; u < NTJ; ++u) acc[u][0] = acc[u][1] = 0.0;
#pragma unroll 4
                for (int k0 = 0; k0 < NBB; k0 += 4) {
                    const double a = Vs[(wr + g) + (k0 + q4) * VLD];
#pragma unroll
                    for (int u = 0; u < NTJ; ++u) nrg::cta_dmma(acc[u][0], acc[u][1], a, Ws[(k0 + q4) * CBK + u * 8 + g]);
                }
#pragma unroll
                for (int u = 0; u < NTJ; ++u) {
                    W2[(wr + g) * CBK + u * 8 + 2 * q4] = acc[u][0];
                    W2[(wr + g) * CBK + u * 8 + 2 * q4 + 1] = acc[u][1];
                }
            } else {
                // Z(r0:, :) -= V W2 on the chunk's 64 rows
                const int i0 = 64 * (t - C - 1), rows = min(64, mr - i0);
#pragma unroll
                for (int u = 0; u < NTJ; ++u) acc[u][0] = acc[u][1] = 0.0;
#pragma unroll 4
                for (int k0 = 0; k0 < NBB; k0 += 4) {
                    const double a = Vs[(k0 + q4) * VLD + wr + g];
#pragma unroll
                    for (int u = 0; u < NTJ; ++u) nrg::cta_dmma(acc[u][0], acc[u][1], a, W2[(k0 + q4) * CBK + u * 8 + g]);
                }
                const int row = wr + g;
                if (row < rows) {
                    double* zr = Zs + r0 + i0 + row;
#pragma unroll
                    for (int u = 0; u < NTJ; ++u) {
                        zr[(size_t)(u * 8 + 2 * q4) * ldz] -= acc[u][0];
                        zr[(size_t)(u * 8 + 2 * q4 + 1) * ldz] -= acc[u][1];
                    }
                }
            }
            __syncthreads();
            buf ^= 1;
        }
    }
    for (int j = 0; j < nc; ++j)
        for (int row = tid; row < n; row += 256)
            L.A[(size_t)row + (size_t)(c0 + j) * n] = Zs[(size_t)j * ldz + row];
}

__global__ void k_large_out(const LSec* __restrict__ secs, double* eigbuf, double* wsd, int* wsi) {
    const LSec sec = secs[blockIdx.y];
    LView L = lview(sec, eigbuf, wsd, wsi);
    const long long n = sec.n, sq = n * n;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < sq; e += (long long)gridDim.x * blockDim.x)
        L.A[e] = L.Z[e];
}

// the eigenvalues (ascending, the divide and conquer's order) to the output, one block
// per sector, as soon as the divide and conquer has finished
__global__ void k_large_evals(const LSec* __restrict__ secs, double* eigbuf, double* evals, double* wsd, int* wsi) {
    const LSec sec = secs[blockIdx.x];
    LView L = lview(sec, eigbuf, wsd, wsi);
    for (int i = threadIdx.x; i < sec.n; i += blockDim.x) evals[sec.e_off + i] = L.D[i];
}

}  // namespace

namespace nrg {

// ---------------------------------------------------------------------------------
// host orchestration
// ---------------------------------------------------------------------------------
// One cluster of kTriCL blocks per sector when the own panel rows fit in shared memory
// and the device can place such a cluster; *done = false leaves the multi-kernel path.
template <int CL>
static int tri_cluster_cl(nrg_context* ctx, const LSec* dsec, int ns, int maxn, double* d_V, double* wsd,
                          int* wsi, bool* done) {
    *done = false;
    TriLayout lay;
    lay.MM = (maxn + CL - 1) / CL;
    lay.PN = maxn + (maxn & 1);
    lay.NRB = (maxn + 511) / 512;
    if (lay.MM > TT) return NRG_OK;
    const size_t smem = sizeof(double) * (size_t)lay.doubles(CL);
    int dev = 0, optin = 0;
    NRG_CUDA_TRY(cudaGetDevice(&dev));
    NRG_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    if (smem > (size_t)optin) return NRG_OK;
    NRG_TRY(raise_smem_limit((const void*)k_tri_cluster<CL>, smem));
    if (CL > 8) NRG_CUDA_TRY(cudaFuncSetAttribute(k_tri_cluster<CL>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(CL * ns));
    cfg.blockDim = dim3(TT);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = ctx->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = CL;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, k_tri_cluster<CL>, &cfg) != cudaSuccess || clusters < 1) {
        cudaGetLastError();
        return NRG_OK;
    }
    NRG_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_tri_cluster<CL>, dsec, lay, d_V, wsd, wsi));
    ctx->launches++;
    *done = true;
    return NRG_OK;
}

// The lower-triangle variant, when its layout fits in shared memory: the column ranges
// of its product are as narrow as the space allows (more work items to balance).
template <int CL>
static int tri_csym_cl(nrg_context* ctx, const LSec* dsec, int ns, int maxn, double* d_V, double* wsd,
                       int* wsi, bool* done) {
    *done = false;
    int dev = 0, optin = 0;
    NRG_CUDA_TRY(cudaGetDevice(&dev));
    NRG_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    TriLayoutS lay;
    lay.MM = (maxn + CL - 1) / CL;
    lay.PN = maxn + (maxn & 1);
    if (lay.MM > TT) return NRG_OK;
    const size_t smem = sizeof(double) * (size_t)lay.doubles(CL);
    if (smem > (size_t)optin) return NRG_OK;
    NRG_TRY(raise_smem_limit((const void*)k_tri_csym<CL>, smem));
    if (CL > 8) NRG_CUDA_TRY(cudaFuncSetAttribute(k_tri_csym<CL>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(CL * ns));
    cfg.blockDim = dim3(TT);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = ctx->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = CL;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, k_tri_csym<CL>, &cfg) != cudaSuccess || clusters < 1) {
        cudaGetLastError();
        return NRG_OK;
    }
    NRG_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_tri_csym<CL>, dsec, lay, d_V, wsd, wsi));
    ctx->launches++;
    *done = true;
    return NRG_OK;
}

// Cluster size of the one-launch tridiagonalisation: 8 blocks per sector (16 for the
// largest size class alone halves its per-block product but costs as much in the wider
// exchanges: no net gain measured); a size that cannot be placed falls back to the next
// smaller one.  The environment variable NRG_TRI_CLUSTER forces 4, 8 or 16, or 0 for the
// multi-kernel path.  NRG_TRI_SYM=1 takes the lower-triangle kernel (8 or 16 blocks) when
// its layout fits: it moves half the bytes but measured slower on the bench workloads
// (23.8 against 16.3 ms per launch at N_keep = 4096: more time at the barriers per column),
// so the full-column kernel is the default.
static int tri_cluster(nrg_context* ctx, const LSec* dsec, int ns, int maxn, double* d_V, double* wsd,
                       int* wsi, bool* done) {
    static const int forced = [] {
        const char* e = getenv("NRG_TRI_CLUSTER");
        if (!e || !*e) return -1;
        const int v = atoi(e);
        return (v == 0 || v == 4 || v == 8 || v == 16) ? v : -1;
    }();
    static const bool sym = [] {
        const char* e = getenv("NRG_TRI_SYM");
        return e && e[0] == '1';
    }();
    // launches whose largest sector reaches this order take 16-block clusters: their
    // column product (the trailing matrix streamed from L2) outweighs the wider exchanges
    static const int cl16_min = [] {
        const char* e = getenv("NRG_TRI_CL16_MIN");
        return (e && *e) ? atoi(e) : kTriCL16Min;
    }();
    *done = false;
    const int cl = forced >= 0 ? forced : (maxn >= cl16_min ? 16 : kTriCL);
    if (sym && cl == 16) {
        NRG_TRY(tri_csym_cl<16>(ctx, dsec, ns, maxn, d_V, wsd, wsi, done));
        if (*done) return NRG_OK;
    }
    if (sym && cl == 8) {
        NRG_TRY(tri_csym_cl<8>(ctx, dsec, ns, maxn, d_V, wsd, wsi, done));
        if (*done) return NRG_OK;
        // orders whose 8-block layout does not fit (above ~1,500) fit on 16-block clusters
        // up to ~2,300
        if (forced < 0) {
            NRG_TRY(tri_csym_cl<16>(ctx, dsec, ns, maxn, d_V, wsd, wsi, done));
            if (*done) return NRG_OK;
        }
    }
    if (cl == 16) {
        NRG_TRY(tri_cluster_cl<16>(ctx, dsec, ns, maxn, d_V, wsd, wsi, done));
        if (*done || forced == 16) return NRG_OK;
    }
    if (cl == 16 && !*done) {   // 16 could not be placed: the 8-block kernel
        NRG_TRY(tri_cluster_cl<8>(ctx, dsec, ns, maxn, d_V, wsd, wsi, done));
        if (*done) return NRG_OK;
    }
    if (cl >= 8) {
        NRG_TRY(tri_cluster_cl<8>(ctx, dsec, ns, maxn, d_V, wsd, wsi, done));
        if (*done || forced == 8) return NRG_OK;
    }
    if (cl >= 4) return tri_cluster_cl<4>(ctx, dsec, ns, maxn, d_V, wsd, wsi, done);
    return NRG_OK;
}

int syev_large(nrg_context* ctx, const std::vector<SyevSector>& in, double* d_V, double* d_E, int slot_base,
               cudaEvent_t evals_ready) {
    const int ns = (int)in.size();
    if (ns == 0) return NRG_OK;
    cudaStream_t st = ctx->stream;
    std::vector<LSec> secs(ns);
    long long wd = 0, wi = 0;
    int maxn = 0;
    for (int s = 0; s < ns; ++s) {
        secs[s].a_off = in[s].a_off;
        secs[s].e_off = in[s].e_off;
        secs[s].n = in[s].n;
        secs[s].pad = 0;
        secs[s].w_off = wd;
        secs[s].i_off = wi;
        wd += lws_doubles(in[s].n);
        wi += lws_ints(in[s].n);
        maxn = std::max(maxn, in[s].n);
    }
    DevBuf& bsec = ctx->scratch.b[slot_base];
    DevBuf& bwd = ctx->scratch.b[slot_base + 1];
    DevBuf& bwi = ctx->scratch.b[slot_base + 2];
    DevBuf& bidx = ctx->scratch.b[slot_base + 3];
    DevBuf& bmrg = ctx->scratch.b[slot_base + 4];
    const int gslot = slot_base + 5;   // grouped GEMM problem lists (two slots)
    NRG_TRY(bsec.ensure(sizeof(LSec) * ns));
    NRG_TRY(bwd.ensure(sizeof(double) * (size_t)wd));
    NRG_TRY(bwi.ensure(sizeof(int) * (size_t)wi));
    NRG_TRY(h2d_async(ctx, bsec.p, secs.data(), sizeof(LSec) * ns));
    const LSec* dsec = bsec.as<LSec>();
    double* wsd = bwd.as<double>();
    int* wsi = bwi.as<int>();
    // column index lists of the panel update [V W] and [W V] for every panel width jc
    {
        std::vector<int> idx(2 * NB * 2 * NB);
        for (int jc = 1; jc <= NB; ++jc)
            for (int q = 0; q < 2 * NB; ++q) {
                idx[(size_t)(jc - 1) * 4 * NB + q] = q < jc ? q : NB + (q - jc);            // [V W]
                idx[(size_t)(jc - 1) * 4 * NB + 2 * NB + q] = q < jc ? NB + q : q - jc;     // [W V]
            }
        NRG_TRY(bidx.ensure(sizeof(int) * idx.size()));
        NRG_TRY(h2d_async(ctx, bidx.p, idx.data(), sizeof(int) * idx.size()));
    }
    const int* didx = bidx.as<int>();
    const size_t symv_smem = sizeof(double) * (size_t)maxn;
    if (symv_smem > 48 * 1024)
        NRG_TRY(raise_smem_limit((const void*)k_tri_symv, symv_smem));

    // ---- 1. tridiagonalisation ----
    bool clustered = false;
    cudaEvent_t te[2] = {nullptr, nullptr};
    if (ctx->profiling) {
        NRG_CUDA_TRY(cudaEventCreate(&te[0]));
        NRG_CUDA_TRY(cudaEventCreate(&te[1]));
        NRG_CUDA_TRY(cudaEventRecord(te[0], st));
    }
    NRG_TRY(tri_cluster(ctx, dsec, ns, maxn, d_V, wsd, wsi, &clustered));
    if (ctx->profiling) {
        NRG_CUDA_TRY(cudaEventRecord(te[1], st));
        if (clustered) {
            nrg_context::PendingTimer t{te[0], te[1], 0.0, 0.0};
            for (int x = 0; x < ns; ++x) {
                const double n = secs[x].n;
                t.flops += 4.0 / 3.0 * n * n * n;
                t.bytes += 8.0 * n * n * n / 3.0;
            }
            ctx->pending_tri.push_back(t);
        } else {
            cudaEventDestroy(te[0]);
            cudaEventDestroy(te[1]);
        }
    }
    for (int p = 0; !clustered && p < maxn - 1; p += NB) {
        for (int j = 0; j < NB; ++j) {
            const int k = p + j;
            if (k > maxn - 2) break;
            k_tri_col<<<ns, TPB, 0, st>>>(dsec, k, d_V, wsd, wsi);
            int nblk = 0;
            for (int s = 0; s < ns; ++s)
                if (k <= secs[s].n - 2) nblk += (secs[s].n - k - 1 + CB - 1) / CB;
            k_tri_symv<<<nblk, TPB, symv_smem, st>>>(dsec, ns, k, d_V, wsd, wsi);
            ctx->launches += 2;
        }
        k_tri_finish<<<ns, TPB, 0, st>>>(dsec, p, d_V, wsd, wsi);
        ctx->launches++;
        NRG_CUDA_TRY(cudaGetLastError());
        std::vector<GemmProblem> probs;
        for (int s = 0; s < ns; ++s) {
            const int n = secs[s].n;
            const int c = std::min(p + NB - 1, n - 2);
            if (c < p) continue;
            const int jc = c - p + 1, r0 = p + jc;
            if (r0 >= n) continue;
            double* VW = wsd + secs[s].w_off + 3LL * n * n;
            GemmProblem P;
            std::memset(&P, 0, sizeof(P));
            P.M = n - r0; P.N = n - r0; P.K = 2 * jc;
            P.alpha = -1.0; P.beta = 1.0;
            P.A = VW + r0; P.a_si = 1; P.a_sk = n; P.a_ki = didx + (size_t)(jc - 1) * 4 * NB;
            P.B = VW + r0; P.b_sk = n; P.b_ki = didx + (size_t)(jc - 1) * 4 * NB + 2 * NB; P.b_sj = 1;
            P.C = d_V + secs[s].a_off + r0 + (long long)r0 * n; P.c_si = 1; P.c_sj = n;
            probs.push_back(P);
        }
        NRG_TRY(launch_ggemm(ctx, probs, gslot));
    }
    if (!clustered) {
        k_tri_end<<<ns, 32, 0, st>>>(dsec, d_V, wsd, wsi);
        ctx->launches++;
    }

    // ---- 2. divide and conquer ----
    {
        const size_t smem = sizeof(double) * (32 + nrg::kCtaGemmSmem + kDcSmemDoubles * DC_LOW);
        int nchunk = 0;
        for (int x = 0; x < ns; ++x) nchunk += (secs[x].n + DC_LOW - 1) / DC_LOW;
        k_dc_low<<<nchunk, 512, smem, st>>>(dsec, ns, d_V, wsd, wsi, ctx->d_status.as<int>());
        ctx->launches++;
        NRG_CUDA_TRY(cudaGetLastError());
    }
    for (int s = DC_LOW; s < maxn; s *= 2) {
        std::vector<Merge> ms;
        int blk[3] = {0, 0, 0};
        for (int x = 0; x < ns; ++x) {
            const int n = secs[x].n;
            for (int a = 0; a + s < n; a += 2 * s) {
                Merge m;
                m.sec = x; m.a = a; m.mid = a + s; m.b = std::min(a + 2 * s, n);
                const long long nn = m.b - m.a;
                m.nblk[kMapItem] = (int)((nn + TPB - 1) / TPB);
                m.nblk[kMapWarp] = (int)((nn * 32 + TPB - 1) / TPB);
                m.nblk[kMapWide] = (int)((nn * nn + (long long)TPB * kWideItems - 1) / ((long long)TPB * kWideItems));
                for (int q = 0; q < 3; ++q) {
                    m.blk0[q] = blk[q];
                    blk[q] += m.nblk[q];
                }
                ms.push_back(m);
            }
        }
        if (ms.empty()) continue;
        const int nm = (int)ms.size();
        NRG_TRY(bmrg.ensure(sizeof(Merge) * nm));
        NRG_TRY(h2d_async(ctx, bmrg.p, ms.data(), sizeof(Merge) * nm));
        const Merge* dms = bmrg.as<Merge>();
        k_dc_prep<<<nm, 512, 0, st>>>(dsec, dms, d_V, wsd, wsi);
        for (int ph = 1; ph <= 4; ++ph)
            k_dc_phase<<<blk[ph <= 3 ? kMapWarp : kMapItem], TPB, 0, st>>>(dsec, dms, nm, ph, d_V, wsd, wsi,
                                                                           ctx->d_status.as<int>());
        k_dc_poscols<<<blk[kMapItem], TPB, 0, st>>>(dsec, dms, nm, d_V, wsd, wsi);
        ctx->launches += 6;
        NRG_CUDA_TRY(cudaGetLastError());
        // the number K of non-deflated roots of each merge stays on the device: the
        // GEMM is launched for K = nn and reads the true K (I[7n + a]) itself
        std::vector<GemmProblem> probs;
        for (int i = 0; i < nm; ++i) {
            const Merge& m = ms[i];
            const int n = secs[m.sec].n, nn = m.b - m.a;
            double* W = wsd + secs[m.sec].w_off;
            const long long sq = (long long)n * n;
            int* I = wsi + secs[m.sec].i_off;
            GemmProblem P;
            std::memset(&P, 0, sizeof(P));
            P.M = nn; P.N = nn; P.K = nn; P.alpha = 1.0; P.beta = 0.0;
            P.dyn_nk = I + 7LL * n + m.a;
            P.A = W + m.a; P.a_si = 1; P.a_sk = n; P.a_ki = I + 5LL * n + m.a;          // Z(:, a+perm[nd[q]])
            P.B = W + sq + m.a + (long long)m.a * n; P.b_sk = 1; P.b_sj = n;           // U block
            P.C = W + 2 * sq + m.a; P.c_si = 1; P.c_sj = n; P.c_ji = I + 6LL * n + m.a;  // Qt(:, a+pos[j])
            probs.push_back(P);
        }
        NRG_TRY(launch_ggemm(ctx, probs, gslot));
        k_dc_phase<<<blk[kMapWide], TPB, 0, st>>>(dsec, dms, nm, 5, d_V, wsd, wsi, ctx->d_status.as<int>());
        k_dc_phase<<<blk[kMapWide], TPB, 0, st>>>(dsec, dms, nm, 6, d_V, wsd, wsi, ctx->d_status.as<int>());
        ctx->launches += 2;
        NRG_CUDA_TRY(cudaGetLastError());
    }

    k_large_evals<<<ns, TPB, 0, st>>>(dsec, d_V, d_E, wsd, wsi);
    ctx->launches++;
    NRG_CUDA_TRY(cudaGetLastError());
    if (evals_ready) NRG_CUDA_TRY(cudaEventRecord(evals_ready, st));

    // ---- 3. back-transformation ----
    // one pass per column block with the block resident in shared memory, when it fits
    {
        int dev = 0, optin = 0;
        NRG_CUDA_TRY(cudaGetDevice(&dev));
        NRG_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        auto apply_smem = [&](int c) {   // Z block (ld up to maxn + 15), two staging buffers, W and W2
            return sizeof(double) * ((size_t)(maxn + 15) * c + 2 * NBB * (NBB + 4) + 2 * NBB * c);
        };
        const size_t prep_smem = sizeof(double) * (NBB * 65 + 2 * NBB * NBB);
        const int cbk = apply_smem(16) <= (size_t)optin ? 16 : (apply_smem(8) <= (size_t)optin ? 8 : 0);
        if (cbk > 0) {
            const int npan = (maxn - 2) / NBB + 1;
            NRG_TRY(raise_smem_limit((const void*)k_bt_prep, prep_smem));
            k_bt_prep<<<dim3(npan, ns), 256, prep_smem, st>>>(dsec, d_V, wsd, wsi);
            int nblk = 0;
            for (int x = 0; x < ns; ++x) nblk += (secs[x].n + cbk - 1) / cbk;
            const size_t sm = apply_smem(cbk);
            if (cbk == 16) {
                NRG_TRY(raise_smem_limit((const void*)k_bt_apply<16>, sm));
                k_bt_apply<16><<<nblk, 256, sm, st>>>(dsec, ns, d_V, wsd, wsi);
            } else {
                NRG_TRY(raise_smem_limit((const void*)k_bt_apply<8>, sm));
                k_bt_apply<8><<<nblk, 256, sm, st>>>(dsec, ns, d_V, wsd, wsi);
            }
            ctx->launches += 2;
            NRG_CUDA_TRY(cudaGetLastError());
            return NRG_OK;
        }
    }
    // otherwise panels of NBB reflectors on grouped GEMMs, last panel first
    const int qmax = (maxn - 2) / NBB;   // panels cover reflectors 0 .. n-2
    const size_t tf_smem = sizeof(double) * 2 * NBB * NBB;
    NRG_TRY(raise_smem_limit((const void*)k_bt_tfactor, tf_smem));
    for (int q = qmax; q >= 0; --q) {
        std::vector<int> act;
        for (int s = 0; s < ns; ++s)
            if (q * NBB < secs[s].n - 1) act.push_back(s);
        if (act.empty()) continue;
        k_bt_vpanel<<<dim3(16, ns), TPB, 0, st>>>(dsec, q, d_V, wsd, wsi);
        ctx->launches++;
        std::vector<GemmProblem> g1;
        for (int s : act) {
            const int n = secs[s].n, nr = n - 1, jb = q * NBB, b = std::min(NBB, nr - jb);
            const int r0 = jb + 1, mr = n - r0;
            double* W = wsd + secs[s].w_off;
            const long long sq = (long long)n * n;
            double* Vb = W + sq;            // U
            double* G = W + 2 * sq;         // Qt: G (NBB x NBB), T, then V^T Z
            GemmProblem P;
            std::memset(&P, 0, sizeof(P));
            P.M = b; P.N = b; P.K = mr; P.alpha = 1.0; P.beta = 0.0;
            P.A = Vb; P.a_si = mr; P.a_sk = 1;
            P.B = Vb; P.b_sk = 1; P.b_sj = mr;
            P.C = G; P.c_si = 1; P.c_sj = NBB;
            g1.push_back(P);
            GemmProblem Q;
            std::memset(&Q, 0, sizeof(Q));
            Q.M = b; Q.N = n; Q.K = mr; Q.alpha = 1.0; Q.beta = 0.0;
            Q.A = Vb; Q.a_si = mr; Q.a_sk = 1;
            Q.B = W + r0; Q.b_sk = 1; Q.b_sj = n;                       // Z(r0:, :)
            Q.C = G + 2 * NBB * NBB; Q.c_si = 1; Q.c_sj = b;            // Wt (b x n)
            g1.push_back(Q);
        }
        NRG_TRY(launch_ggemm(ctx, g1, gslot));
        k_bt_tfactor<<<ns, NBB, tf_smem, st>>>(dsec, q, d_V, wsd, wsi);
        ctx->launches++;
        std::vector<GemmProblem> g2, g3;
        for (int s : act) {
            const int n = secs[s].n, nr = n - 1, jb = q * NBB, b = std::min(NBB, nr - jb);
            const int r0 = jb + 1, mr = n - r0;
            double* W = wsd + secs[s].w_off;
            const long long sq = (long long)n * n;
            double* Vb = W + sq;
            double* Tm = W + 2 * sq + NBB * NBB;
            double* Wt = W + 2 * sq + 2 * NBB * NBB;
            double* VT = Vb + (long long)mr * NBB;     // (mr x b) after Vb in U
            GemmProblem P;
            std::memset(&P, 0, sizeof(P));
            P.M = mr; P.N = b; P.K = b; P.alpha = 1.0; P.beta = 0.0;
            P.A = Vb; P.a_si = 1; P.a_sk = mr;
            P.B = Tm; P.b_sk = 1; P.b_sj = NBB;
            P.C = VT; P.c_si = 1; P.c_sj = mr;
            g2.push_back(P);
            GemmProblem Q;
            std::memset(&Q, 0, sizeof(Q));
            Q.M = mr; Q.N = n; Q.K = b; Q.alpha = -1.0; Q.beta = 1.0;
            Q.A = VT; Q.a_si = 1; Q.a_sk = mr;
            Q.B = Wt; Q.b_sk = 1; Q.b_sj = b;
            Q.C = W + r0; Q.c_si = 1; Q.c_sj = n;
            g3.push_back(Q);
        }
        NRG_TRY(launch_ggemm(ctx, g2, gslot));
        NRG_TRY(launch_ggemm(ctx, g3, gslot));
    }
    k_large_out<<<dim3(32, ns), TPB, 0, st>>>(dsec, d_V, wsd, wsi);
    ctx->launches++;
    NRG_CUDA_TRY(cudaGetLastError());
    return NRG_OK;
}

}  // namespace nrg
