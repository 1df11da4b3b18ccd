// Batched FP64 symmetric eigensolver for the symmetry-sector blocks of one NRG
// iteration (the dsyev('V','U') call of diagonalization.F90:267, one call per sector),
// one thread block per sector.  Used for blocks of order <= 128 (large blocks go through
// the multi-kernel pipeline of eig_large.cu, which reuses the pieces below):
//   1. Householder tridiagonalisation of the lower triangle (H = Q T Q^T), in shared
//      memory for orders <= 128, reflectors kept in the block's own storage;
//   2. divide and conquer on T (Cuppen tearing down to 1x1 leaves, deflation of small
//      z components and of close pole pairs by Givens rotations, secular roots by a
//      safeguarded rational iteration in pole-shifted coordinates, Gu-Eisenstat
//      recomputation of z for orthogonal eigenvectors); merges of up to 32 rows run one
//      per warp, larger merges use the whole block and an in-block tiled GEMM;
//   3. back-transformation V = Q Z with 32 reflectors at a time (compact WY form,
//      two in-block GEMMs per panel).
// Eigenvalues come out ascending with their eigenvectors in the same column order, as
// dsyev returns them.
#include "eig_common.cuh"
#include "internal.hpp"

namespace {

constexpr int kThreads = 512;
constexpr int kNB = 32;           // reflectors per back-transform panel
constexpr int kSmemTri = 128;     // orders tridiagonalised in shared memory
constexpr int kDcCap = 128;       // orders whose divide and conquer vectors live in shared memory

// Householder tridiagonalisation of the n x n block A (leading dim lda, full storage kept
// symmetric); reflector k is stored below the subdiagonal of column k with an implicit 1.
__device__ void tridiagonalise(double* A, int lda, int n, double* Dd, double* Ee, double* TAU,
                               double* vs, double* ps, double* red) {
    const int tid = threadIdx.x, T = blockDim.x;
    for (int k = 0; k < n - 1; ++k) {
        const int m = n - k - 1;
        double* col = A + (size_t)k * lda;
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
            const double* Ai = A + (size_t)(k + 1 + i) + (size_t)(k + 1) * lda;
            double s0 = 0.0, s1 = 0.0;
            int j = 0;
            for (; j + 1 < m; j += 2) {
                s0 = fma(Ai[(size_t)j * lda], vs[j], s0);
                s1 = fma(Ai[(size_t)(j + 1) * lda], vs[j + 1], s1);
            }
            if (j < m) s0 = fma(Ai[(size_t)j * lda], vs[j], s0);
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
            double* Aj = A + (size_t)(k + 1) + (size_t)(k + 1 + j) * lda;
            for (int i = tid; i < m; i += T) Aj[i] -= vs[i] * wj + ps[i] * vj;
        }
        __syncthreads();
    }
    for (int k = tid; k < n; k += T) Dd[k] = A[(size_t)k + (size_t)k * lda];
    if (tid == 0) Ee[n - 1] = 0.0;
    __syncthreads();
}

// back-transformation Z <- Q Z with Q = H_0 ... H_{n-2} (reflectors in A), kNB at a time
__device__ void back_transform(const double* A, int n, const double* TAU, double* Z, double* Vb,
                               double* Qt, double* Ts, double* Gs, double* gsm) {
    const int tid = threadIdx.x, T = blockDim.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int nr = n - 1;
    for (int jb = ((nr - 1) / kNB) * kNB; jb >= 0; jb -= kNB) {
        const int b = min(kNB, nr - jb);
        const int r0 = jb + 1, mr = n - r0;
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
                double acc = 0.0;
                if (lane < c)
                    for (int q = lane; q < c; ++q) acc += Ts[lane + q * kNB] * (-tc * Gs[q + c * kNB]);
                __syncwarp();
                if (lane < c) Ts[lane + c * kNB] = acc;
                if (lane == 0) Ts[c + c * kNB] = tc;
                __syncwarp();
            }
        }
        __syncthreads();
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
}

__global__ void __launch_bounds__(kThreads) k_syev(const SyevSector* __restrict__ secs,
                                                    double* __restrict__ eigbuf,
                                                    double* __restrict__ evals,
                                                    double* __restrict__ wsd, int* __restrict__ wsi,
                                                    int* status, int smem_tri) {
    extern __shared__ double sm[];
    const SyevSector sec = secs[blockIdx.x];
    const int n = sec.n;
    const int tid = threadIdx.x, T = blockDim.x;
    double* A = eigbuf + sec.a_off;
    double* ev = evals + sec.e_off;
    {
        // a block holding NaN or Inf is reported and left undiagonalised (its eigenvalues
        // become NaN): the iterations below have fixed bounds, but their results would
        // be meaningless
        bool bad = false;
        for (long long e = tid; e < (long long)n * n; e += T) bad |= !isfinite(A[e]);
        if (__syncthreads_or(bad)) {
            if (tid == 0) atomicOr(status, NRG_DEV_NONFINITE);
            for (int i = tid; i < n; i += T) ev[i] = __longlong_as_double(0x7ff8000000000000LL);
            return;
        }
    }
    if (n == 1) {
        if (tid == 0) { ev[0] = A[0]; A[0] = 1.0; }
        return;
    }
    double* W = wsd + sec.w_off;
    const long long sq = (long long)n * n;
    double* Z = W;
    double* U = W + sq;
    double* Qt = W + 2 * sq;
    const long long qt = sq > 64LL * n ? sq : 64LL * n;
    double* vec = W + 2 * sq + qt;
    double* Dd = vec;
    double* Ee = vec + n;
    double* TAU = vec + 2 * n;
    int* I = wsi + sec.i_off;
    Scratch S = scratch_at(vec, I, n);

    double* red = sm;
    double* gsm = sm + 32;
    double* vs = sm + 32 + nrg::kCtaGemmSmem;
    const int vlen = n > kNB * kNB ? n : kNB * kNB;
    double* ps = vs + vlen;
    double* dcs = vs + 2 * vlen + kNB * kNB;          // D and the merge vectors (orders <= kDcCap)
    double* As = dcs + kDcSmemDoubles * kDcCap;

    // ---- 1. tridiagonalisation ----
    if (smem_tri && n <= kSmemTri) {
        for (long long e = tid; e < sq; e += T) As[e] = A[e];
        __syncthreads();
        tridiagonalise(As, n, n, Dd, Ee, TAU, vs, ps, red);
        for (long long e = tid; e < sq; e += T) A[e] = As[e];
        __syncthreads();
    } else {
        tridiagonalise(A, n, n, Dd, Ee, TAU, vs, ps, red);
    }

    // ---- 2. divide and conquer on (Dd, Ee) -> eigenvalues in Dm, vectors in Z ----
    double* Dm = Dd;
    Scratch Sm = S;
    if (n <= kDcCap) {
        Dm = dcs;
        Sm = scratch_smem(dcs, kDcCap);
    }
    for (long long e = tid; e < sq; e += T) Z[e] = 0.0;
    __syncthreads();
    for (int i = tid; i < n; i += T) {
        Z[(size_t)i + (size_t)i * n] = 1.0;
        double dv = Dd[i];
        if (i > 0) dv -= fabs(Ee[i - 1]);
        if (i < n - 1) dv -= fabs(Ee[i]);
        Dm[i] = dv;
    }
    __syncthreads();
    const int warp = tid >> 5, lane = tid & 31, nwarps = T >> 5;
    for (int s = 1; s < n; s *= 2) {
        if (2 * s <= 32) {
            WarpG wg{lane};
            int mi = 0;
            for (int a = 0; a + s < n; a += 2 * s, ++mi) {
                if (mi % nwarps != warp) continue;
                dc_merge(wg, a, a + s, min(a + 2 * s, n), n, Z, Dm, Ee, Sm, U, Qt, red, gsm, status);
            }
            __syncthreads();
        } else {
            BlockG bg;
            for (int a = 0; a + s < n; a += 2 * s)
                dc_merge(bg, a, a + s, min(a + 2 * s, n), n, Z, Dm, Ee, Sm, U, Qt, red, gsm, status);
        }
    }
    __syncthreads();

    // ---- 3. back-transformation ----
    back_transform(A, n, TAU, Z, U, Qt, vs, vs + kNB * kNB, gsm);

    for (int i = tid; i < n; i += T) ev[i] = Dm[i];
    for (long long e = tid; e < sq; e += T) A[e] = Z[e];
}

}  // namespace

int launch_syev(const SyevSector* d_secs, int nsec, int max_n, double* eigbuf, double* evals,
                double* wsd, int* wsi, int* d_status, cudaStream_t st) {
    if (nsec == 0) return NRG_OK;
    const size_t vlen = (size_t)(max_n > kNB * kNB ? max_n : kNB * kNB);
    const int smem_tri = max_n <= kSmemTri ? 1 : 0;
    size_t smem = sizeof(double) * (32 + nrg::kCtaGemmSmem + 2 * vlen + kNB * kNB + kDcSmemDoubles * kDcCap +
                                    (smem_tri ? (size_t)max_n * max_n : 0));
    if (smem > 227 * 1024) {
        nrg_set_error_message("sector of order %d exceeds the shared-memory plan", max_n);
        return NRG_ERR_TOO_LARGE;
    }
    if (smem > 48 * 1024) NRG_TRY(nrg::raise_smem_limit((const void*)k_syev, smem));
    k_syev<<<nsec, kThreads, smem, st>>>(d_secs, eigbuf, evals, wsd, wsi, d_status, smem_tri);
    NRG_CUDA_TRY(cudaGetLastError());
    return NRG_OK;
}
