// Shared definitions for the NRG hot-path kernels (sm_100a, FP64).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <cstdio>

#include "../../include/nrg_b200.h"

#define NRG_CUDA_TRY(expr)                                                        \
    do {                                                                          \
        cudaError_t _e = (expr);                                                  \
        if (_e != cudaSuccess) {                                                  \
            nrg_set_error_message("%s:%d %s -> %s", __FILE__, __LINE__, #expr,    \
                                  cudaGetErrorString(_e));                        \
            return NRG_ERR_CUDA;                                                  \
        }                                                                         \
    } while (0)

#define NRG_TRY(expr)                       \
    do {                                    \
        int _s = (expr);                    \
        if (_s != NRG_OK) return _s;        \
    } while (0)

void nrg_set_error_message(const char* fmt, ...);

// device status flags written by kernels (bit set; read back by the host)
enum : int {
    NRG_DEV_OK = 0,
    NRG_DEV_BAD_INDEX = 1,       // a gathered index fell outside its array
    NRG_DEV_SMEM = 2,            // a block did not fit the configured shared memory
    NRG_DEV_SECULAR = 4,         // a secular root did not bracket
    NRG_DEV_NONFINITE = 8,       // NaN/Inf met in an input block
};

// --------------------------------------------------------------------------------------
// eigensolver work description (one entry per symmetry sector)
// --------------------------------------------------------------------------------------
struct SyevSector {
    long long a_off;    // offset of the d x d block in the eigenvector buffer
    long long w_off;    // offset of the double workspace
    long long i_off;    // offset of the int workspace
    long long e_off;    // offset of the eigenvalues (start_input - 1)
    int n;
    int pad;
};

// double workspace per sector of order n
__host__ __device__ inline long long syev_ws_doubles(long long n) {
    long long sq = n * n;
    long long qt = sq > 64 * n ? sq : 64 * n;
    return 2 * sq + qt + 16 * n + 64;
}
__host__ __device__ inline long long syev_ws_ints(long long n) { return 12 * n + 64; }

// launch helpers implemented in the .cu files (return NRG status)
int launch_syev(const SyevSector* d_secs, int nsec, int max_n, double* eigbuf, double* evals,
                double* wsd, int* wsi, int* d_status, cudaStream_t st);
