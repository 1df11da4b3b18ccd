// nrg_block_eigh_noalloc: the per-sector FP64 eigensolver of nrg_diagonalization for one
// symmetric block, for callers that cannot allocate device memory.  Its workspace lives in
// the file-scope device array below (allocated when the library is loaded on a device and
// held until the process exits); the call itself allocates nothing.
#include "common.cuh"

#include <cuda.h>   // CUcontext and CUresult only: driver calls go through cudaGetDriverEntryPoint

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

// The array's device address, looked up once per device and CUDA context.  The address
// belongs to the context the library's device code was loaded into: after the application
// resets the device (cudaDeviceReset) a new primary context loads the module again, and
// the old address is stale.  The context is told apart by its process-unique id
// (cuCtxGetId, through the runtime's driver entry points: no link against libcuda).
struct ScratchEntry {
    unsigned long long ctx_id;   // 0: unknown, look up again on the next call
    double* ptr;
};
ScratchEntry g_scratch[kMaxDevices] = {};

typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);

// id of the calling thread's current context; 0 when there is none or it cannot be told
unsigned long long current_context_id() {
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static bool resolved = false;
    if (!resolved) {   // under g_mu
        resolved = true;
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<CtxGetCurrentFn>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<CtxGetIdFn>(f);
        cudaGetLastError();
    }
    if (!get_current || !get_id) return 0;
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (get_current(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// device address of the static array on the current device
int scratch_address(int device, double** out) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (device < 0 || device >= kMaxDevices) return NRG_ERR_DEVICE;
    ScratchEntry& e = g_scratch[device];
    unsigned long long id = current_context_id();
    if (e.ptr && id != 0 && id == e.ctx_id) {
        *out = e.ptr;
        return NRG_OK;
    }
    void* p = nullptr;
    const cudaError_t err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (err != cudaSuccess) {
        nrg_set_error_message("cudaGetSymbolAddress of the static workspace failed: %s", cudaGetErrorString(err));
        return NRG_ERR_CUDA;
    }
    if (id == 0) id = current_context_id();   // the lookup made the primary context current
    e.ptr = static_cast<double*>(p);
    e.ctx_id = id;
    *out = e.ptr;
    return NRG_OK;
}

// memory this device's kernels may read and write: device memory of the current device,
// or managed memory; a device pointer of another GPU is refused (no peer access is set up)
bool on_device(const void* p, int device) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (a.type == cudaMemoryTypeManaged) return true;
    return a.type == cudaMemoryTypeDevice && a.device == device;
}

}  // namespace

extern "C" int nrg_block_eigh_noalloc(const double* H, int32_t n, double* eigenvalues,
                                      double* eigenvectors, void* stream) {
    if (n < 1 || n > kMaxN) {
        nrg_set_error_message("nrg_block_eigh_noalloc: order %d outside 1..%lld (the static workspace limit)",
                              n, kMaxN);
        return NRG_ERR_TOO_LARGE;
    }
    int device = 0;
    NRG_CUDA_TRY(cudaGetDevice(&device));
    if (!H || !eigenvalues || !eigenvectors || !on_device(H, device) || !on_device(eigenvalues, device) ||
        !on_device(eigenvectors, device)) {
        nrg_set_error_message("nrg_block_eigh_noalloc: H, eigenvalues and eigenvectors must be device arrays "
                              "of the current device (%d) or managed memory", device);
        return NRG_ERR_INVALID;
    }
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
