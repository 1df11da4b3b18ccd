// nrg_block_eigh_noalloc: the per-sector FP64 eigensolver of nrg_diagonalization for one
// symmetric block, for callers that cannot allocate device memory.  Its workspace lives in
// the file-scope device array below (allocated when the library is loaded on a device and
// held until the process exits); the call itself allocates nothing.
#include "common.cuh"

#include <mutex>

namespace {

// largest block order the static workspace covers
constexpr long long kMaxN = NRG_NOALLOC_MAX_ORDER;
constexpr long long kWsDoubles = 2 * kMaxN * kMaxN + (kMaxN * kMaxN > 64 * kMaxN ? kMaxN * kMaxN : 64 * kMaxN) +
                                 16 * kMaxN + 64;
constexpr long long kWsInts = 12 * kMaxN + 64;
constexpr long long kIntsAsDoubles = (kWsInts + 1) / 2;
// [0, 8): sector descriptor, [8, 16): status word, then the int and double workspaces
constexpr long long kDescOff = 0, kStatusOff = 8, kIntOff = 16, kDblOff = kIntOff + kIntsAsDoubles;
constexpr long long kTotalDoubles = kDblOff + kWsDoubles;
static_assert(sizeof(SyevSector) <= 8 * sizeof(double), "descriptor slot too small");

}  // namespace

// the workspace: one copy per device that loads the library (~417 KB), kept until exit
static __device__ __align__(256) double g_noalloc_scratch[kTotalDoubles];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_ptr[kMaxDevices] = {nullptr};

// device address of the static array on the current device (set up once per device)
int scratch_address(int device, double** out) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (device < 0 || device >= kMaxDevices) return NRG_ERR_DEVICE;
    if (!g_scratch_ptr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            nrg_set_error_message("cudaGetSymbolAddress of the static workspace failed: %s", cudaGetErrorString(e));
            return NRG_ERR_CUDA;
        }
        g_scratch_ptr[device] = static_cast<double*>(p);
    }
    *out = g_scratch_ptr[device];
    return NRG_OK;
}

bool on_device(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace

extern "C" int nrg_block_eigh_noalloc(const double* H, int32_t n, double* eigenvalues,
                                      double* eigenvectors, void* stream) {
    if (n < 1 || n > kMaxN) {
        nrg_set_error_message("nrg_block_eigh_noalloc: order %d outside 1..%lld (the static workspace limit)",
                              n, kMaxN);
        return NRG_ERR_TOO_LARGE;
    }
    if (!H || !eigenvalues || !eigenvectors || !on_device(H) || !on_device(eigenvalues) ||
        !on_device(eigenvectors)) {
        nrg_set_error_message("nrg_block_eigh_noalloc: H, eigenvalues and eigenvectors must be device arrays");
        return NRG_ERR_INVALID;
    }
    int device = 0;
    NRG_CUDA_TRY(cudaGetDevice(&device));
    double* base = nullptr;
    NRG_TRY(scratch_address(device, &base));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    SyevSector sec;
    sec.a_off = 0;
    sec.w_off = 0;
    sec.i_off = 0;
    sec.e_off = 0;
    sec.n = n;
    sec.pad = 0;
    SyevSector* d_sec = reinterpret_cast<SyevSector*>(base + kDescOff);
    int* d_status = reinterpret_cast<int*>(base + kStatusOff);
    int* d_ints = reinterpret_cast<int*>(base + kIntOff);
    double* d_ws = base + kDblOff;
    // the workspace keeps the previous call's contents: the status word must start at zero;
    // the eigensolver writes every other workspace entry before reading it
    NRG_CUDA_TRY(cudaMemsetAsync(d_status, 0, sizeof(int), st));
    NRG_CUDA_TRY(cudaMemcpyAsync(d_sec, &sec, sizeof(sec), cudaMemcpyHostToDevice, st));
    if (eigenvectors != H)
        NRG_CUDA_TRY(cudaMemcpyAsync(eigenvectors, H, sizeof(double) * (size_t)n * n, cudaMemcpyDeviceToDevice, st));
    NRG_TRY(launch_syev(d_sec, 1, n, eigenvectors, eigenvalues, d_ws, d_ints, d_status, st));
    int flags = 0;
    NRG_CUDA_TRY(cudaMemcpyAsync(&flags, d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
    NRG_CUDA_TRY(cudaStreamSynchronize(st));
    if (flags != 0) {
        nrg_set_error_message("nrg_block_eigh_noalloc: device status flags 0x%x", flags);
        return NRG_ERR_NUMERIC;
    }
    return NRG_OK;
}
