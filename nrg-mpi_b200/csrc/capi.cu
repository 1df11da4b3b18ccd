// C ABI entry points (include/nrg_b200.h): context, model, and the drop-in replacements
// of the reference routines.  Host arrays are staged through device buffers; device
// arrays are used in place.
#include "internal.hpp"

#include <algorithm>
#include <chrono>
#include <cstdarg>
#include <cstdlib>
#include <cstring>
#include <execinfo.h>
#include <initializer_list>
#include <signal.h>
#include <unistd.h>
#include <unordered_set>
#include <vector>

namespace {
thread_local char g_err[1024] = "";

// NRG_SEGV_TRACE=1: print the native call stack on a host crash, then hand the signal to
// the previous handler (diagnostics only)
struct sigaction g_prev_segv;
char g_altstack[1 << 16];
void segv_trace(int sig, siginfo_t* si, void* uc) {
    static const char msg[] = "\n[nrg] SIGSEGV, native stack:\n";
    if (write(2, msg, sizeof(msg) - 1) < 0) {}
    void* buf[64];
    const int n = backtrace(buf, 64);
    backtrace_symbols_fd(buf, n, 2);
    sigaction(SIGSEGV, &g_prev_segv, nullptr);
    if (g_prev_segv.sa_flags & SA_SIGINFO) {
        if (g_prev_segv.sa_sigaction) g_prev_segv.sa_sigaction(sig, si, uc);
    } else if (g_prev_segv.sa_handler != SIG_DFL && g_prev_segv.sa_handler != SIG_IGN) {
        g_prev_segv.sa_handler(sig);
    }
    signal(sig, SIG_DFL);
    raise(sig);
}
__attribute__((constructor)) void install_segv_trace() {
    const char* e = getenv("NRG_SEGV_TRACE");
    if (!e || e[0] != '1') return;
    void* warm[4];
    backtrace(warm, 4);   // loads the unwinder outside the handler
    stack_t ss;
    ss.ss_sp = g_altstack;
    ss.ss_size = sizeof(g_altstack);
    ss.ss_flags = 0;
    sigaltstack(&ss, nullptr);
    struct sigaction sa;
    memset(&sa, 0, sizeof(sa));
    sa.sa_sigaction = segv_trace;
    sa.sa_flags = SA_SIGINFO | SA_ONSTACK;
    sigemptyset(&sa.sa_mask);
    sigaction(SIGSEGV, &sa, &g_prev_segv);
}
}

void nrg_set_error_message(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

nrg_context::~nrg_context() {
    for (auto& b : store) b.release();
    for (auto& b : host_store) b.release();
    for (auto& b : scratch.b) b.release();
    for (auto& s : iter_sectors) { s.d_bi.release(); s.d_lst.release(); s.d_lstOff.release(); }
    for (auto& t : table_pool) { t.bi.release(); t.lst.release(); t.off.release(); }
    d_status.release();
    nrg::Model& M = model;
    for (nrg::DevBuf* b : {&M.d_operation, &M.d_dflag, &M.d_dtype, &M.d_dch, &M.d_dswp, &M.d_bflag,
                           &M.d_bch, &M.d_dcoef, &M.d_imflag, &M.d_imcoef})
        b->release();
    for (auto& c : stage_inflight) {
        cudaEventSynchronize(c.ev);
        cudaEventDestroy(c.ev);
    }
    for (cudaEvent_t e : event_pool) cudaEventDestroy(e);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (aux) cudaStreamDestroy(aux);
    if (ev_join2) cudaEventDestroy(ev_join2);
    if (aux2) cudaStreamDestroy(aux2);
    if (ev_join_hi) cudaEventDestroy(ev_join_hi);
    for (cudaEvent_t e : {ev_evals_hi, ev_evals2, ev_evals_host})
        if (e) cudaEventDestroy(e);
    h_small.release();
    h_evals.release();
    h_kept.release();
    if (aux_hi) cudaStreamDestroy(aux_hi);
    if (aux_copy) cudaStreamDestroy(aux_copy);
    if (ev_copied) cudaEventDestroy(ev_copied);
    for (auto* pl : {&pending_tri, &pending_syev})
        for (auto& t : *pl) {
            cudaEventDestroy(t.a);
            cudaEventDestroy(t.b);
        }
    if (stage_host) cudaFreeHost(stage_host);
}

using namespace nrg;

namespace {

bool is_device_ptr(const void* p) {
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Every entry point checks its arrays first: device memory must belong to the context's
// device (the library sets up no peer access, so a kernel reading another GPU's memory
// would fault); host memory of any kind and managed memory are accepted.
int reject_foreign(const nrg_context* ctx, const char* who, std::initializer_list<const void*> ptrs) {
    int k = 0;
    for (const void* p : ptrs) {
        ++k;
        if (!p) continue;
        cudaPointerAttributes a;
        if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
            cudaGetLastError();
            continue;
        }
        if (a.type == cudaMemoryTypeDevice && a.device != ctx->device) {
            nrg_set_error_message("%s: array %d is memory of device %d, the context runs on device %d", who, k,
                                  a.device, ctx->device);
            return NRG_ERR_INVALID;
        }
    }
    return NRG_OK;
}

// Host wall-clock parts of one drop-in entry call with profiling on: the stream is drained
// at each mark, so the staging copies, the device work and the copies out are timed apart
struct EntryClock {
    nrg_context* ctx;
    bool on;
    std::chrono::steady_clock::time_point t;
    explicit EntryClock(nrg_context* c) : ctx(c), on(c->profiling) {
        if (!on) return;
        cudaStreamSynchronize(ctx->stream);
        t = std::chrono::steady_clock::now();
        ++ctx->entry_calls;
    }
    void mark(int part) {
        if (!on) return;
        cudaStreamSynchronize(ctx->stream);
        const auto n = std::chrono::steady_clock::now();
        ctx->entry_s[part] += std::chrono::duration<double>(n - t).count();
        t = n;
    }
};

// A drop-in call's Sectors takes the device table buffers of pool slot k before its upload
// and gives them back (grown, if they grew) when the call ends; the swap leaves the other
// side empty
void swap_tables(nrg_context* ctx, Sectors& S, size_t k) {
    nrg_context::TableBufs& t = ctx->table_slot(k);
    std::swap(S.d_bi, t.bi);
    std::swap(S.d_lst, t.lst);
    std::swap(S.d_lstOff, t.off);
}

template <class T>
int stage_in(nrg_context* ctx, const T* p, size_t n, size_t slot, const T** out) {
    if (n == 0) { *out = nullptr; return NRG_OK; }
    if (!p) { nrg_set_error_message("NULL input array"); return NRG_ERR_INVALID; }
    if (is_device_ptr(p)) { *out = p; return NRG_OK; }
    DevBuf& b = ctx->slot(slot);
    NRG_TRY(b.ensure(sizeof(T) * n));
    NRG_CUDA_TRY(cudaMemcpyAsync(b.p, p, sizeof(T) * n, cudaMemcpyHostToDevice, ctx->stream));
    ctx->h2d += (long long)(sizeof(T) * n);
    *out = b.as<T>();
    return NRG_OK;
}

constexpr size_t kSlotIO = 100000;   // drop-in staging slots

// stage_in for an input of which the routine reads only the listed runs: pinned host
// memory is read run by run by a kernel (only those bytes cross the host link, the
// rest of the device copy is never read); from pageable memory the runs are gathered on
// the host into a page-locked buffer, copied in one piece and scattered to their places
// on the device (the whole array is copied instead when the runs are most of it)
int stage_in_pageable_segs(nrg_context* ctx, const double* p, size_t n, long long ld,
                           const std::vector<HostSeg>& segs, size_t slot, const double** out) {
    long long total = 0;
    for (const auto& g : segs) total += (long long)g.len * g.count;
    if (total == 0 || 2 * total > (long long)n) return stage_in(ctx, p, n, slot, out);
    for (const auto& g : segs)
        if (g.len < 0 || g.count < 0 || g.off < 0 || g.off + (long long)(g.count - 1) * ld + g.len > (long long)n) {
            nrg_set_error_message("segment outside the input array");
            return NRG_ERR_INVALID;
        }
    HostBuf& h = ctx->seg_slot(slot - kSlotIO);
    NRG_TRY(h.ensure(sizeof(double) * (size_t)total));
    double* pk = h.as<double>();
    long long at = 0;
    for (const auto& g : segs)
        for (int r = 0; r < g.count; ++r) {
            std::memcpy(pk + at, p + g.off + (long long)r * ld, sizeof(double) * (size_t)g.len);
            at += g.len;
        }
    DevBuf& b = ctx->slot(slot);
    DevBuf& bp = ctx->slot(slot + 50000);
    NRG_TRY(b.ensure(sizeof(double) * n));
    NRG_TRY(bp.ensure(sizeof(double) * (size_t)total));
    NRG_CUDA_TRY(cudaMemcpyAsync(bp.p, pk, sizeof(double) * (size_t)total, cudaMemcpyHostToDevice, ctx->stream));
    long long bytes = 0;
    NRG_TRY(run_gather_segs(ctx, bp.as<double>(), b.as<double>(), ld, segs, &bytes, true));
    ctx->h2d += bytes;
    *out = b.as<double>();
    // the page-locked buffer is rewritten by the next call on this slot: the copy must
    // have left it (the drop-in entries drain the stream before they return as well)
    NRG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return NRG_OK;
}

int stage_in_segs(nrg_context* ctx, const double* p, size_t n, long long ld, const std::vector<HostSeg>& segs,
                  size_t slot, const double** out) {
    if (n == 0) { *out = nullptr; return NRG_OK; }
    if (!p) { nrg_set_error_message("NULL input array"); return NRG_ERR_INVALID; }
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return stage_in_pageable_segs(ctx, p, n, ld, segs, slot, out);
    }
    if (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) { *out = p; return NRG_OK; }
    if (a.type != cudaMemoryTypeHost || !a.devicePointer) return stage_in_pageable_segs(ctx, p, n, ld, segs, slot, out);
    DevBuf& b = ctx->slot(slot);
    NRG_TRY(b.ensure(sizeof(double) * n));
    long long bytes = 0;
    NRG_TRY(run_gather_segs(ctx, static_cast<const double*>(a.devicePointer), b.as<double>(), ld, segs, &bytes));
    ctx->h2d += bytes;
    *out = b.as<double>();
    return NRG_OK;
}

template <class T>
int stage_out(nrg_context* ctx, T* p, size_t n, size_t slot, T** dev) {
    if (!p) { nrg_set_error_message("NULL output array"); return NRG_ERR_INVALID; }
    if (is_device_ptr(p)) { *dev = p; return NRG_OK; }
    DevBuf& b = ctx->slot(slot);
    NRG_TRY(b.ensure(sizeof(T) * std::max<size_t>(n, 1)));
    *dev = b.as<T>();
    return NRG_OK;
}

template <class T>
int finish_out(nrg_context* ctx, T* p, const T* dev, size_t n) {
    if (p == dev || n == 0) return NRG_OK;
    NRG_CUDA_TRY(cudaMemcpyAsync(p, dev, sizeof(T) * n, cudaMemcpyDeviceToHost, ctx->stream));
    ctx->d2h += (long long)(sizeof(T) * n);
    return NRG_OK;
}

template <class T>
std::vector<T> to_host(nrg_context* ctx, const T* p, size_t n, int* status) {
    std::vector<T> v(n);
    *status = NRG_OK;
    if (n == 0) return v;
    if (is_device_ptr(p)) {
        cudaError_t e = cudaMemcpyAsync(v.data(), p, sizeof(T) * n, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) { *status = NRG_ERR_CUDA; nrg_set_error_message("%s", cudaGetErrorString(e)); }
    } else {
        std::memcpy(v.data(), p, sizeof(T) * n);
    }
    return v;
}

int need_model(nrg_context* ctx) {
    if (!ctx) { nrg_set_error_message("NULL context"); return NRG_ERR_INVALID; }
    if (!ctx->model.set) { nrg_set_error_message("nrg_context_set_model has not been called"); return NRG_ERR_STATE; }
    return NRG_OK;
}

template <class T>
int up(DevBuf& b, const std::vector<T>& v, cudaStream_t st) {
    NRG_TRY(b.ensure(sizeof(T) * std::max<size_t>(v.size(), 1)));
    if (!v.empty()) NRG_CUDA_TRY(cudaMemcpyAsync(b.p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, st));
    return NRG_OK;
}


}  // namespace

extern "C" {

const char* nrg_last_error(void) { return g_err; }

const char* nrg_status_string(int s) {
    switch (s) {
        case NRG_OK: return "ok";
        case NRG_ERR_INVALID: return "invalid argument";
        case NRG_ERR_CUDA: return "CUDA error";
        case NRG_ERR_NOMEM: return "out of device memory";
        case NRG_ERR_TOO_LARGE: return "block too large";
        case NRG_ERR_DEVICE: return "no usable CUDA device";
        case NRG_ERR_UNSUPPORTED: return "unsupported input";
        case NRG_ERR_STATE: return "call sequence error";
        case NRG_ERR_NUMERIC: return "numerical failure";
        case NRG_ERR_TIMEOUT: return "device wait timed out";
        default: return "unknown status";
    }
}

int nrg_version(void) { return 1; }

int nrg_context_create(nrg_context** out, int device) {
    if (!out) return NRG_ERR_INVALID;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= device || device < 0) {
        cudaGetLastError();
        nrg_set_error_message("no CUDA device %d (count %d)", device, n);
        return NRG_ERR_DEVICE;
    }
    NRG_CUDA_TRY(cudaSetDevice(device));
    cudaDeviceProp prop;
    NRG_CUDA_TRY(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10) {
        nrg_set_error_message("device %d is sm_%d%d; this library is built for sm_100a", device, prop.major, prop.minor);
        return NRG_ERR_DEVICE;
    }
    nrg_context* c = new nrg_context();
    c->device = device;
    int st = c->d_status.ensure(sizeof(int) * 4);
    if (st != NRG_OK) { delete c; return st; }
    if (cudaMemset(c->d_status.p, 0, sizeof(int) * 4) != cudaSuccess) { delete c; return NRG_ERR_CUDA; }
    *out = c;
    return NRG_OK;
}

int nrg_context_destroy(nrg_context* ctx) {
    if (!ctx) return NRG_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    delete ctx;
    return NRG_OK;
}

int nrg_context_set_stream(nrg_context* ctx, void* stream) {
    if (!ctx) return NRG_ERR_INVALID;
    ctx->stream = (cudaStream_t)stream;
    return NRG_OK;
}

int64_t nrg_context_launch_count(const nrg_context* ctx) { return ctx ? ctx->launches : 0; }

int nrg_context_get_stats(const nrg_context* ctx, nrg_stats* out) {
    if (!ctx || !out) return NRG_ERR_INVALID;
    out->launches = ctx->launches;
    out->syev_launches = ctx->syev_launches;
    out->syev_ms = ctx->syev_ms;
    out->syev_flops = ctx->syev_flops;
    out->h2d_bytes = ctx->h2d;
    out->d2h_bytes = ctx->d2h;
    out->tri_launches = ctx->tri_launches;
    out->tri_ms = ctx->tri_ms;
    out->tri_flops = ctx->tri_flops;
    out->tri_bytes = ctx->tri_bytes;
    out->entry_in_s = ctx->entry_s[0];
    out->entry_compute_s = ctx->entry_s[1];
    out->entry_out_s = ctx->entry_s[2];
    out->entry_calls = ctx->entry_calls;
    out->replay_host_s = ctx->replay_host_s;
    return NRG_OK;
}

int nrg_context_reset_stats(nrg_context* ctx) {
    if (!ctx) return NRG_ERR_INVALID;
    NRG_TRY(flush_profile_timers(ctx));   // timers of an unfinished run are dropped below
    ctx->syev_launches = 0;
    ctx->syev_ms = 0.0;
    ctx->syev_flops = 0.0;
    ctx->h2d = 0;
    ctx->d2h = 0;
    ctx->tri_launches = 0;
    ctx->tri_ms = ctx->tri_flops = ctx->tri_bytes = 0.0;
    ctx->entry_s[0] = ctx->entry_s[1] = ctx->entry_s[2] = 0.0;
    ctx->entry_calls = 0;
    ctx->replay_host_s = 0.0;
    return NRG_OK;
}

int nrg_host_alloc(size_t bytes, void** out) {
    if (!out) return NRG_ERR_INVALID;
    *out = nullptr;
    if (bytes == 0) return NRG_OK;
    cudaError_t e = cudaHostAlloc(out, bytes, cudaHostAllocPortable);
    if (e != cudaSuccess) {
        *out = nullptr;
        nrg_set_error_message("cudaHostAlloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
        return NRG_ERR_NOMEM;
    }
    return NRG_OK;
}

int nrg_host_free(void* p) {
    if (!p) return NRG_OK;
    NRG_CUDA_TRY(cudaFreeHost(p));
    return NRG_OK;
}

int nrg_context_release_storage(nrg_context* ctx) {
    if (!ctx) return NRG_ERR_INVALID;
    NRG_CUDA_TRY(cudaSetDevice(ctx->device));
    NRG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    for (auto& b : ctx->store) b.release();
    ctx->store.clear();
    for (auto& b : ctx->host_store) b.release();
    ctx->host_store.clear();
    for (auto& b : ctx->scratch.b) b.release();
    for (auto& s : ctx->iter_sectors) { s.d_bi.release(); s.d_lst.release(); s.d_lstOff.release(); }
    ctx->iter_sectors.clear();
    for (auto& t : ctx->table_pool) { t.bi.release(); t.lst.release(); t.off.release(); }
    ctx->table_pool.clear();
    return NRG_OK;
}

int nrg_context_set_profiling(nrg_context* ctx, int on) {
    if (!ctx) return NRG_ERR_INVALID;
    ctx->profiling = on != 0;
    return NRG_OK;
}

int nrg_context_set_model(nrg_context* ctx, const nrg_model* m) {
    if (!ctx || !m) return NRG_ERR_INVALID;
    NRG_CUDA_TRY(cudaSetDevice(ctx->device));
    Model& M = ctx->model;
    M.set = false;
    M.nIter = m->numberOfIteration; M.nChain = m->numberOfChain; M.nVar = m->numberOfVariation;
    for (int i = 0; i < 4; ++i) M.cb[i] = m->conservationBlock[i];
    M.nMat = m->flag_spectrum ? m->numberOfMatrix : 0;
    M.nCM = m->numberOfConductionMatrix; M.nCoef = m->numberOfCoefficient;
    M.nOps = m->numberOfOperation; M.nBCS = m->numberOfBCSCoefficient;
    M.first = m->indexOfFirstIteration; M.flag_spectrum = m->flag_spectrum; M.flag_BCS = m->flag_BCS;
    M.D = m->bandWidth; M.z = m->ztrick; M.Lambda = m->Lambda;
    M.scalingType = m->scalingType; M.truncation = m->truncation;
    if (M.nVar < 1 || M.nOps < 1 || M.nChain < 1 || M.nCM < 1 || M.nIter < M.first || M.nCoef < 0) {
        nrg_set_error_message("inconsistent model sizes");
        return NRG_ERR_INVALID;
    }
    if (!m->operation || (M.nCoef > 0 && (!m->coefficient_invariant_matrix_type ||
        !m->coefficient_invariant_matrix || !m->coefficient_diagonalization_type ||
        !m->coefficient_diagonalization)) || !m->chain_diagonal || !m->chain_nondiagonal) {
        nrg_set_error_message("missing model table");
        return NRG_ERR_INVALID;
    }
    const int nOps = M.nOps, nVar = M.nVar, nChain = M.nChain;
    M.operation.assign(m->operation, m->operation + (size_t)nOps * (nVar + nChain));
    const size_t nd = (size_t)(M.nIter + 2) * nChain, nn = (size_t)(M.nIter + 2 - M.first) * nChain;
    M.chain_diag.assign(m->chain_diagonal, m->chain_diagonal + nd);
    M.chain_nond.assign(m->chain_nondiagonal, m->chain_nondiagonal + nn);
    M.chain_bcs.clear();
    if (M.flag_BCS && m->chain_BCS) M.chain_bcs.assign(m->chain_BCS, m->chain_BCS + nd);
    if (M.nMat > 0) {
        if (!m->coefficient_invariant_matrix_spectrum || !m->conservation_difference_spectrum ||
            !m->positiveSpectrumOperation || !m->negativeSpectrumOperation) {
            nrg_set_error_message("missing spectrum table");
            return NRG_ERR_INVALID;
        }
        M.cspec.assign(m->coefficient_invariant_matrix_spectrum, m->coefficient_invariant_matrix_spectrum + (size_t)M.nMat * nOps);
        M.cons_diff.assign(m->conservation_difference_spectrum, m->conservation_difference_spectrum + (size_t)M.nMat * nVar);
        M.pos_op.assign(m->positiveSpectrumOperation, m->positiveSpectrumOperation + (size_t)M.nMat * nVar);
        M.neg_op.assign(m->negativeSpectrumOperation, m->negativeSpectrumOperation + (size_t)M.nMat * nVar);
    }
    // coefficient scans of diagonalization.F90:195-224 and invariantMatrixDGEMM.F90:248-254
    const int nC = M.nCoef;
    auto cdt = [&](int ic, int col) { return m->coefficient_diagonalization_type[(size_t)ic + (size_t)col * nC]; };
    auto cit = [&](int ic, int col) { return m->coefficient_invariant_matrix_type[(size_t)ic + (size_t)col * nC]; };
    const size_t nn2 = (size_t)nOps * nOps;
    M.dflag.assign(nn2, 0); M.dtype.assign(nn2, 0); M.dch.assign(nn2, 0); M.dswp.assign(nn2, 0);
    M.dcoef.assign(nn2, 0.0); M.bflag.assign(nn2, 0); M.bch.assign(nn2, 0);
    for (int a = 1; a <= nOps; ++a)
        for (int b = 1; b <= nOps; ++b) {
            const size_t x = (size_t)(a - 1) * nOps + (b - 1);
            for (int ic = 0; ic < nC; ++ic) {
                if (a == cdt(ic, 0) && b == cdt(ic, 1)) {
                    M.dflag[x] = 1; M.dtype[x] = cdt(ic, 2); M.dch[x] = cdt(ic, 3);
                    M.dcoef[x] = m->coefficient_diagonalization[ic];
                } else if (a == cdt(ic, 1) && b == cdt(ic, 0)) {
                    M.dflag[x] = 1; M.dtype[x] = cdt(ic, 2); M.dch[x] = cdt(ic, 3);
                    M.dcoef[x] = m->coefficient_diagonalization[ic];
                    M.dswp[x] = 1;
                }
            }
            if (M.dflag[x] && (M.dtype[x] < 1 || M.dtype[x] > M.nCM || M.dch[x] < 1 || M.dch[x] > nChain)) {
                nrg_set_error_message("coefficient_diagonalization_type row out of range");
                return NRG_ERR_INVALID;
            }
        }
    if (M.flag_BCS && m->coefficient_BCS) {
        for (int ic = 0; ic < M.nBCS; ++ic) {
            const int a = m->coefficient_BCS[ic], b = m->coefficient_BCS[ic + M.nBCS], ch = m->coefficient_BCS[ic + 2 * M.nBCS];
            if (a < 1 || a > nOps || b < 1 || b > nOps) return NRG_ERR_INVALID;
            const size_t x = (size_t)(a - 1) * nOps + (b - 1);
            M.bflag[x] = 1; M.bch[x] = ch;
        }
    }
    M.imflag.assign(nn2 * M.nCM, 0);
    M.imcoef.assign(nn2 * M.nCM, 0.0);
    for (int ic = 0; ic < nC; ++ic) {
        const int a = cit(ic, 0), b = cit(ic, 1), t = cit(ic, 2);
        if (a < 1 || a > nOps || b < 1 || b > nOps || t < 1 || t > M.nCM) {
            nrg_set_error_message("coefficient_invariant_matrix_type row out of range");
            return NRG_ERR_INVALID;
        }
        const size_t x = ((size_t)(a - 1) * nOps + (b - 1)) * M.nCM + (t - 1);
        M.imflag[x] = 1;
        M.imcoef[x] = m->coefficient_invariant_matrix[ic];
    }
    cudaStream_t st = ctx->stream;
    NRG_TRY(up(M.d_operation, M.operation, st));
    NRG_TRY(up(M.d_dflag, M.dflag, st)); NRG_TRY(up(M.d_dtype, M.dtype, st));
    NRG_TRY(up(M.d_dch, M.dch, st)); NRG_TRY(up(M.d_dswp, M.dswp, st));
    NRG_TRY(up(M.d_dcoef, M.dcoef, st)); NRG_TRY(up(M.d_bflag, M.bflag, st));
    NRG_TRY(up(M.d_bch, M.bch, st)); NRG_TRY(up(M.d_imflag, M.imflag, st));
    NRG_TRY(up(M.d_imcoef, M.imcoef, st));
    NRG_CUDA_TRY(cudaStreamSynchronize(st));
    M.set = true;
    return NRG_OK;
}

// ------------------------------------------------------------------------------------
int nrg_diagonalization(nrg_context* ctx, int32_t iteration, const nrg_diagonalization_io* io) {
    NRG_TRY(need_model(ctx));
    if (!io) return NRG_ERR_INVALID;
    NRG_CUDA_TRY(cudaSetDevice(ctx->device));
    NRG_TRY(reject_foreign(ctx, "nrg_diagonalization",
                           {io->subspaceInfo, io->basis_input, io->eigenvalue_old, io->invariant_matrix, io->eigenvalue,
                            io->eigenvector, io->basis_output, io->groundStateEnergy}));
    EntryClock clk(ctx);
    const Model& M = ctx->model;
    if (iteration < M.first || iteration > M.nIter) {
        nrg_set_error_message("iteration %d outside [%d, %d]", iteration, M.first, M.nIter);
        return NRG_ERR_INVALID;
    }
    const int rs = M.nVar + 3;
    int st = NRG_OK;
    auto si = to_host(ctx, io->subspaceInfo, (size_t)io->numberOfSubspace * rs, &st);
    NRG_TRY(st);
    auto bi = to_host(ctx, io->basis_input, (size_t)io->numberOfBasis * rs, &st);
    NRG_TRY(st);
    Sectors S;
    swap_tables(ctx, S, 0);
    int rc = S.build(io->numberOfSubspace, si.data(), io->numberOfBasis, bi.data(), M.nVar, M.nOps);
    if (rc == NRG_OK) rc = S.upload(ctx);
    if (rc != NRG_OK) { swap_tables(ctx, S, 0); return rc; }
    const int nbo = io->numberOfBasis_old;
    if (io->sizeOfEigenvector < S.sizeV || nbo < 1) {
        nrg_set_error_message("eigenvector capacity %lld < %lld", (long long)io->sizeOfEigenvector, S.sizeV);
        rc = NRG_ERR_INVALID;
    }
    const double *dEo = nullptr, *dIM = nullptr;
    double *dV = nullptr, *dE = nullptr;
    if (rc == NRG_OK) rc = stage_in(ctx, io->eigenvalue_old, (size_t)nbo, kSlotIO + 0, &dEo);
    if (rc == NRG_OK) {
        // the blocks of invariant_matrix the assembly reads (diagonalization.F90:195-237):
        // for every ordered pair of operation groups of a sector whose coefficient scan
        // found a term, the previous-sector rows of one group against the columns of the
        // other (IM(jref, iref, type), swapped as the scan says)
        std::vector<HostSeg> segs;
        std::unordered_set<long long> seen;   // segments already listed
        const int nOps = M.nOps;
        for (int s = 0; s < S.nsub; ++s)
            for (int a = 0; a < nOps; ++a) {
                const int ca = S.cnt(s, a);
                if (ca == 0) continue;
                for (int b = 0; b < nOps; ++b) {
                    const int cb = S.cnt(s, b);
                    const int idx = a * nOps + b;
                    if (cb == 0 || !M.dflag[idx]) continue;
                    const int t = M.dtype[idx] - 1;
                    if (t < 0 || t >= M.nCM) continue;
                    const int ra = S.refBase[(size_t)s * nOps + a], rb = S.refBase[(size_t)s * nOps + b];
                    const bool sw = M.dswp[idx] != 0;
                    const int r0 = sw ? ra : rb, nr = sw ? ca : cb, c0 = sw ? rb : ra, nc = sw ? cb : ca;
                    if (r0 < 0 || c0 < 0 || r0 + nr > nbo || c0 + nc > nbo) continue;   // the kernel flags it
                    const long long key = ((long long)t * nbo + c0) * nbo + r0;
                    if (!seen.insert(key).second) continue;
                    segs.push_back({r0 + (long long)c0 * nbo + (long long)t * nbo * nbo, nr, nc});
                }
            }
        rc = stage_in_segs(ctx, io->invariant_matrix, (size_t)nbo * nbo * M.nCM, nbo, segs, kSlotIO + 1, &dIM);
    }
    if (rc == NRG_OK) rc = stage_out(ctx, io->eigenvector, (size_t)S.sizeV, kSlotIO + 2, &dV);
    if (rc == NRG_OK) rc = stage_out(ctx, io->eigenvalue, (size_t)S.nb, kSlotIO + 3, &dE);
    DiagOut out;
    // a page-locked eigenvector array takes each group's blocks as soon as they are final
    DiagPost post;
    if (rc == NRG_OK && dV != io->eigenvector) {
        cudaPointerAttributes a;
        if (cudaPointerGetAttributes(&a, io->eigenvector) == cudaSuccess && a.type == cudaMemoryTypeHost)
            post.h_V = io->eigenvector;
        cudaGetLastError();
    }
    clk.mark(0);
    if (rc == NRG_OK) rc = diag_device(ctx, iteration, S, dEo, nbo, dIM, dV, dE, &out, &post);
    clk.mark(1);
    if (rc == NRG_OK && !post.copied_V) rc = finish_out(ctx, io->eigenvector, dV, (size_t)S.sizeV);
    if (rc == NRG_OK) rc = finish_out(ctx, io->eigenvalue, dE, (size_t)S.nb);
    if (rc == NRG_OK && io->basis_output) {
        std::vector<int> bo((size_t)S.nb * rs, 0);
        for (int s = 0; s < S.nsub; ++s)
            for (int j = 0; j < S.dim[s]; ++j) {
                int* r = &bo[(size_t)(S.start[s] + j) * rs];
                for (int v = 0; v < M.nVar; ++v) r[v] = S.qn[(size_t)s * M.nVar + v];
                r[M.nVar] = j + 1;
            }
        if (is_device_ptr(io->basis_output))
            rc = cudaMemcpyAsync(io->basis_output, bo.data(), sizeof(int) * bo.size(), cudaMemcpyHostToDevice, ctx->stream) == cudaSuccess ? NRG_OK : NRG_ERR_CUDA;
        else
            std::memcpy(io->basis_output, bo.data(), sizeof(int) * bo.size());
    }
    if (rc == NRG_OK && io->groundStateEnergy) *io->groundStateEnergy = out.groundStateEnergy;
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess && rc == NRG_OK) rc = NRG_ERR_CUDA;
    clk.mark(2);
    swap_tables(ctx, S, 0);
    return rc;
}

static int invmat_common(nrg_context* ctx, int32_t iteration, const nrg_invariant_matrix_io* io, bool spec) {
    NRG_TRY(need_model(ctx));
    if (!io) return NRG_ERR_INVALID;
    NRG_CUDA_TRY(cudaSetDevice(ctx->device));
    NRG_TRY(reject_foreign(ctx, spec ? "nrg_invariant_matrix_for_spectrum_dgemm" : "nrg_invariant_matrix_dgemm",
                           {io->subspaceInfo, io->basis_input, io->basis_output, io->eigenvector,
                            io->invariant_matrix_spectrum_old, io->invariant_matrix}));
    EntryClock clk(ctx);
    const Model& M = ctx->model;
    (void)iteration;
    if (spec && M.nMat == 0) { nrg_set_error_message("model has no spectrum tables"); return NRG_ERR_STATE; }
    const int rs = M.nVar + 3;
    int st = NRG_OK;
    auto si = to_host(ctx, io->subspaceInfo, (size_t)io->numberOfSubspace * rs, &st);
    NRG_TRY(st);
    auto bi = to_host(ctx, io->basis_input, (size_t)io->numberOfBasisFull * rs, &st);
    NRG_TRY(st);
    auto bo = to_host(ctx, io->basis_output, (size_t)io->numberOfBasis * rs, &st);
    NRG_TRY(st);
    Sectors S;
    swap_tables(ctx, S, 0);
    int rc = S.build(io->numberOfSubspace, si.data(), io->numberOfBasisFull, bi.data(), M.nVar, M.nOps);
    if (rc == NRG_OK) rc = S.upload(ctx);
    std::vector<int> kept;
    if (rc == NRG_OK) {
        kept = kept_per_sector(S, io->numberOfBasis, bo.data());
        long long tot = 0;
        for (int s = 0; s < S.nsub; ++s) { tot += kept[s]; if (kept[s] > S.dim[s]) rc = NRG_ERR_INVALID; }
        if (tot != io->numberOfBasis) rc = NRG_ERR_INVALID;
        if (rc != NRG_OK) nrg_set_error_message("kept states do not match the sectors");
    }
    if (rc == NRG_OK && io->sizeOfEigenvector < S.sizeV) rc = NRG_ERR_INVALID;
    const double* dV = nullptr;
    const double* dIMSo = nullptr;
    double* dOut = nullptr;
    const int nbk = io->numberOfBasis;
    const size_t nout = (size_t)nbk * nbk * (spec ? M.nMat : M.nCM);
    if (rc == NRG_OK) {
        // both transforms read the kept columns of each eigenvector block only
        // (invariantMatrixDGEMM.F90:300-317, invariantMatrixForSpectrumDGEMM.F90:296-313)
        std::vector<HostSeg> segs;
        for (int s = 0; s < S.nsub; ++s)
            if (kept[s] > 0) segs.push_back({S.ce[s], S.dim[s] * kept[s], 1});
        rc = stage_in_segs(ctx, io->eigenvector, (size_t)S.sizeV, 0, segs, kSlotIO + 4, &dV);
    }
    if (rc == NRG_OK && spec) {
        // blocks of the previous d-dagger matrix the propagation reads: for each allowed
        // (L, R, m) and local operation a, the previous sectors of (R, a) x (L, a)
        // (invariantMatrixForSpectrumDGEMM.F90:166-256)
        const long long nbo = io->numberOfBasis_old;
        const int nOps = M.nOps, nVar = M.nVar;
        std::vector<HostSeg> segs;
        std::unordered_set<long long> seen;   // segments already listed
        for (int L = 0; L < S.nsub; ++L) {
            if (kept[L] == 0) continue;
            for (int R = 0; R < S.nsub; ++R) {
                if (kept[R] == 0) continue;
                for (int m = 0; m < M.nMat; ++m) {
                    bool ok = true;
                    for (int v = 0; v < nVar && ok; ++v)
                        ok = S.qn[(size_t)L * nVar + v] - S.qn[(size_t)R * nVar + v] ==
                             M.cons_diff[(size_t)m + (size_t)v * M.nMat];
                    if (!ok) continue;
                    for (int a = 0; a < nOps; ++a) {
                        const int cL = S.cnt(L, a), cR = S.cnt(R, a);
                        if (cL == 0 || cR == 0) continue;
                        const long long r0 = S.refBase[(size_t)R * nOps + a], c0 = S.refBase[(size_t)L * nOps + a];
                        if (r0 < 0 || c0 < 0 || r0 + cR > nbo || c0 + cL > nbo) continue;   // rejected below
                        const long long key = ((long long)m * nbo + c0) * nbo + r0;
                        if (!seen.insert(key).second) continue;
                        segs.push_back({r0 + c0 * nbo + (long long)m * nbo * nbo, cR, cL});
                    }
                }
            }
        }
        rc = stage_in_segs(ctx, io->invariant_matrix_spectrum_old, (size_t)(nbo * nbo * M.nMat), nbo, segs,
                           kSlotIO + 5, &dIMSo);
    }
    if (rc == NRG_OK) rc = stage_out(ctx, io->invariant_matrix, nout, kSlotIO + 6, &dOut);
    clk.mark(0);
    if (rc == NRG_OK) {
        if (spec) {
            OpView old;
            old.dense = dIMSo;
            old.nb = io->numberOfBasis_old;
            rc = invmat_spec_device(ctx, S, kept, dV, old, dOut, nullptr, nullptr);
        }
        else rc = invmat_device(ctx, S, kept, dV, dOut);
    }
    clk.mark(1);
    if (rc == NRG_OK) rc = finish_out(ctx, io->invariant_matrix, dOut, nout);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess && rc == NRG_OK) rc = NRG_ERR_CUDA;
    clk.mark(2);
    if (rc == NRG_OK) rc = check_device_status(ctx);
    swap_tables(ctx, S, 0);
    return rc;
}

int nrg_invariant_matrix_dgemm(nrg_context* ctx, int32_t iteration, const nrg_invariant_matrix_io* io) {
    return invmat_common(ctx, iteration, io, false);
}
int nrg_invariant_matrix_for_spectrum_dgemm(nrg_context* ctx, int32_t iteration,
                                            const nrg_invariant_matrix_io* io) {
    return invmat_common(ctx, iteration, io, true);
}

}  // extern "C"

// ------------------------------------------------------------------------------------
// the full stock (fullSubspaceInfo & co.) as per-iteration sector tables
// ------------------------------------------------------------------------------------
namespace {

struct FullIter {
    Sectors S;
    std::vector<int> kept;
    std::vector<long long> rdm_off;
    std::vector<int> rows;      // fullSubspaceInfo row index per sector
};

// builds the sectors of one iteration from rows [r0, r1) of fullSubspaceInfo, its device
// tables in pool slot k (given back by swap_tables(ctx, out->S, k))
int build_full_iter(nrg_context* ctx, const int* fsi, int r0, int r1, const int* fbi, long long nfbi,
                    FullIter* out, size_t k) {
    swap_tables(ctx, out->S, k);
    const Model& M = ctx->model;
    const int nVar = M.nVar, rsf = nVar + 6, rs = nVar + 3;
    const int nsub = r1 - r0;
    std::vector<int> si((size_t)nsub * rs), bi;
    int rowpos = 0;
    out->kept.assign(nsub, 0);
    out->rdm_off.assign(nsub, -1);
    out->rows.resize(nsub);
    std::vector<long long> ce(nsub);
    for (int s = 0; s < nsub; ++s) {
        const int* f = fsi + (size_t)(r0 + s) * rsf;
        const int d = f[nVar], k = f[nVar + 1];
        const long long sin0 = (long long)f[nVar + 3] - 1;
        if (sin0 < 0 || sin0 + d > nfbi) { nrg_set_error_message("fullSubspaceInfo start_input out of range"); return NRG_ERR_INVALID; }
        for (int v = 0; v < nVar; ++v) si[(size_t)s * rs + v] = f[v];
        si[(size_t)s * rs + nVar] = d;
        si[(size_t)s * rs + nVar + 1] = 0;   // replaced below
        si[(size_t)s * rs + nVar + 2] = rowpos + 1;
        bi.insert(bi.end(), fbi + sin0 * rs, fbi + (sin0 + d) * rs);
        rowpos += d;
        out->kept[s] = k;
        out->rdm_off[s] = (long long)f[nVar + 5] - 1;
        out->rows[s] = r0 + s;
        ce[s] = (long long)f[nVar + 2] - 1;
    }
    // count_eigenvector as the running square sums (checked by build), then the stock's
    // start_eigen replaces it: the stock keeps only the kept columns of each block
    long long acc = 0;
    for (int s = 0; s < nsub; ++s) {
        si[(size_t)s * rs + nVar + 1] = (int)std::min(acc + 1, 0x7fffffffLL);
        acc += (long long)si[(size_t)s * rs + nVar] * si[(size_t)s * rs + nVar];
    }
    NRG_TRY(out->S.build(nsub, si.data(), rowpos, bi.data(), nVar, M.nOps));
    out->S.ce = ce;
    return out->S.upload(ctx);
}

int full_range(const int* map, int nIter, int first, int elementNum, int N, int* r0, int* r1) {
    // mapFullSubspaceInfo(-1:nIter), element 0 = iteration -1
    (void)first;
    *r0 = map[N + 1] - 1;
    *r1 = (N == nIter) ? elementNum : map[N + 2] - 1;
    if (*r0 < 0 || *r1 < *r0 || *r1 > elementNum) {
        nrg_set_error_message("mapFullSubspaceInfo inconsistent at iteration %d", N);
        return NRG_ERR_INVALID;
    }
    return NRG_OK;
}

}  // namespace

extern "C" {

int nrg_reduced_density_matrix(nrg_context* ctx, const nrg_reduced_density_io* io) {
    NRG_TRY(need_model(ctx));
    if (!io) return NRG_ERR_INVALID;
    NRG_CUDA_TRY(cudaSetDevice(ctx->device));
    NRG_TRY(reject_foreign(ctx, "nrg_reduced_density_matrix",
                           {io->mapFullSubspaceInfo, io->fullSubspaceInfo, io->fullBasisInput, io->fullBasisOutput,
                            io->fullEigenvector, io->reducedDensityMatrix, io->pointReducedDensity, io->trace}));
    EntryClock clk(ctx);
    const Model& M = ctx->model;
    const int nVar = M.nVar, rsf = nVar + 6, rs = nVar + 3;
    const int nIter = io->numberOfIteration, start = io->startTrancation;
    if (nIter - start <= 0) return NRG_OK;   // reducedDensityMatrixDGEMM.F90:62 loop is empty
    int st = NRG_OK;
    auto map = to_host(ctx, io->mapFullSubspaceInfo, (size_t)(nIter + 2), &st);
    NRG_TRY(st);
    auto fsi = to_host(ctx, (const int*)io->fullSubspaceInfo, (size_t)io->elementNumFullSubspace * rsf, &st);
    NRG_TRY(st);
    auto fbi = to_host(ctx, io->fullBasisInput, (size_t)io->numFullBasisInput * rs, &st);
    NRG_TRY(st);
    const double *dV = nullptr;
    double* dR = nullptr;
    NRG_TRY(stage_in(ctx, io->fullEigenvector, (size_t)io->numFullEigenvector, kSlotIO + 7, &dV));
    NRG_TRY(stage_out(ctx, io->reducedDensityMatrix, (size_t)io->sizeOfReducedDensity, kSlotIO + 8, &dR));
    if (dR != io->reducedDensityMatrix)
        NRG_CUDA_TRY(cudaMemcpyAsync(dR, io->reducedDensityMatrix, sizeof(double) * io->sizeOfReducedDensity,
                                     cudaMemcpyHostToDevice, ctx->stream));
    int point = *io->pointReducedDensity;
    DevBuf& tr = ctx->scratch.b[21];
    NRG_TRY(tr.ensure(sizeof(double) * (size_t)(nIter - start + 1)));
    FullIter child, present;
    size_t sc = 0;   // the table pool slot of child's tables; present's is 1 - sc
    bool has_child = false, has_present = false;
    int rc = NRG_OK;
    int r0, r1;
    clk.mark(0);
    rc = full_range(map.data(), nIter, M.first, io->elementNumFullSubspace, nIter, &r0, &r1);
    if (rc == NRG_OK) {
        rc = build_full_iter(ctx, fsi.data(), r0, r1, fbi.data(), io->numFullBasisInput, &child, sc);
        has_child = true;
    }
    for (int i = 1; rc == NRG_OK && i <= nIter - start; ++i) {
        const int N = nIter - i;
        rc = full_range(map.data(), nIter, M.first, io->elementNumFullSubspace, N, &r0, &r1);
        if (rc != NRG_OK) break;
        // start_matrix of the present iteration (:94-100)
        for (int j = r0; j < r1; ++j) {
            fsi[(size_t)j * rsf + nVar + 5] = point;
            point += fsi[(size_t)j * rsf + nVar + 1] * fsi[(size_t)j * rsf + nVar + 1];
        }
        if (point - 1 > io->sizeOfReducedDensity) { rc = NRG_ERR_INVALID; nrg_set_error_message("reducedDensityMatrix too small"); break; }
        rc = build_full_iter(ctx, fsi.data(), r0, r1, fbi.data(), io->numFullBasisInput, &present, 1 - sc);
        has_present = true;
        if (rc != NRG_OK) break;
        IterView P, C;
        P.S = &present.S; P.kept = present.kept; P.d_V = dV; P.d_rdm = dR; P.rdm_off = present.rdm_off;
        C.S = &child.S; C.kept = child.kept; C.d_V = dV; C.d_rdm = dR; C.rdm_off = child.rdm_off;
        rc = rdm_step_device(ctx, P, C, dR, tr.as<double>() + (i - 1));
        // child's tables back to the pool (the launches that read them precede, on the
        // stream, the uploads of the next borrower); present becomes the child
        swap_tables(ctx, child.S, sc);
        child = present;
        present = FullIter();
        has_present = false;
        sc = 1 - sc;
    }
    if (has_child) swap_tables(ctx, child.S, sc);
    if (has_present) swap_tables(ctx, present.S, 1 - sc);
    clk.mark(1);
    if (rc == NRG_OK) rc = finish_out(ctx, io->reducedDensityMatrix, dR, (size_t)io->sizeOfReducedDensity);
    if (rc == NRG_OK && io->trace) {
        std::vector<double> t(nIter - start);
        NRG_CUDA_TRY(cudaMemcpyAsync(t.data(), tr.p, sizeof(double) * t.size(), cudaMemcpyDeviceToHost, ctx->stream));
        NRG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        std::memcpy(io->trace, t.data(), sizeof(double) * t.size());
    }
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess && rc == NRG_OK) rc = NRG_ERR_CUDA;
    if (rc == NRG_OK) {
        if (is_device_ptr(io->fullSubspaceInfo))
            NRG_CUDA_TRY(cudaMemcpy(io->fullSubspaceInfo, fsi.data(), sizeof(int) * fsi.size(), cudaMemcpyHostToDevice));
        else
            std::memcpy(io->fullSubspaceInfo, fsi.data(), sizeof(int) * fsi.size());
        *io->pointReducedDensity = point;
        rc = check_device_status(ctx);
    }
    clk.mark(2);
    return rc;
}

static int spike_common(nrg_context* ctx, int32_t iteration, const nrg_spike_io* io, bool cfs) {
    NRG_TRY(need_model(ctx));
    if (!io) return NRG_ERR_INVALID;
    NRG_CUDA_TRY(cudaSetDevice(ctx->device));
    NRG_TRY(reject_foreign(ctx, cfs ? "nrg_spike_cfs" : "nrg_spike_zero_temperature",
                           {io->subspaceInfo, io->basis_input, io->basis_output, io->eigenvalue, io->eigenvector,
                            io->invariant_matrix_spectrum, io->fullSubspaceInfo, io->mapFullSubspaceInfo,
                            io->reducedDensityMatrix, io->binnedSpikePositive, io->binnedSpikeNegative,
                            io->total_sum}));
    EntryClock clk(ctx);
    const Model& M = ctx->model;
    if (M.nMat == 0) { nrg_set_error_message("model has no spectrum tables"); return NRG_ERR_STATE; }
    const int nVar = M.nVar, rs = nVar + 3, rsf = nVar + 6;
    const int nbin = M.numberOfBin();
    if (io->numberOfBin != nbin) {
        nrg_set_error_message("numberOfBin %d, expected %d", io->numberOfBin, nbin);
        return NRG_ERR_INVALID;
    }
    int st = NRG_OK;
    const int nbf = io->numberOfBasisFull;
    auto si = to_host(ctx, io->subspaceInfo, (size_t)io->numberOfSubspace * rs, &st); NRG_TRY(st);
    auto bi = to_host(ctx, io->basis_input, (size_t)nbf * rs, &st); NRG_TRY(st);
    auto bo = to_host(ctx, io->basis_output, (size_t)nbf * rs, &st); NRG_TRY(st);
    auto E = to_host(ctx, io->eigenvalue, (size_t)nbf, &st); NRG_TRY(st);
    Sectors S;
    swap_tables(ctx, S, 0);
    int rc = S.build(io->numberOfSubspace, si.data(), nbf, bi.data(), nVar, M.nOps);
    if (rc == NRG_OK) rc = S.upload(ctx);
    if (rc != NRG_OK) { swap_tables(ctx, S, 0); return rc; }
    // eigenvalues back in sector order (the caller's array is in the truncation order)
    std::vector<double> Esec(nbf, 0.0);
    for (int i = 0; i < nbf; ++i) {
        const int s = S.find(&bo[(size_t)i * rs]);
        const int col = bo[(size_t)i * rs + nVar] - 1;
        if (s < 0 || col < 0 || col >= S.dim[s]) { rc = NRG_ERR_INVALID; nrg_set_error_message("basis_output(%d) not in a sector", i + 1); break; }
        Esec[S.start[s] + col] = E[i];
    }
    IterView it;
    it.S = &S;
    it.kept = kept_per_sector(S, io->numberOfBasis, bo.data());
    it.rdm_off.assign(S.nsub, -1);
    std::vector<int> gs;
    if (rc == NRG_OK && cfs) {
        auto map = to_host(ctx, io->mapFullSubspaceInfo, (size_t)(M.nIter + 2), &st); NRG_TRY(st);
        auto fsi = to_host(ctx, io->fullSubspaceInfo, (size_t)io->elementNumFullSubspace * rsf, &st); NRG_TRY(st);
        int r0, r1;
        rc = full_range(map.data(), M.nIter, M.first, io->elementNumFullSubspace, iteration, &r0, &r1);
        for (int j = r0; rc == NRG_OK && j < r1; ++j) {
            const int* f = &fsi[(size_t)j * rsf];
            const int s = S.find(f);
            if (s < 0) continue;
            if (f[nVar] != S.dim[s]) {   // calculateSpectrumDGEMM.F90:418-423
                nrg_set_error_message("variation in fullSubspaceInfo and subspaceInfo is different");
                rc = NRG_ERR_INVALID;
                break;
            }
            it.kept[s] = f[nVar + 1];
            it.rdm_off[s] = (long long)f[nVar + 5] - 1;
        }
    } else if (rc == NRG_OK) {
        for (int i = 0; i < io->numberOfBasis; ++i)
            if (E[i] < 1.0e-8) gs.push_back(S.find(&bo[(size_t)i * rs]));   // :56-75
    }
    const double *dV = nullptr, *dIMS = nullptr, *dR = nullptr;
    double *dEs = nullptr;
    if (rc == NRG_OK) rc = stage_in(ctx, io->eigenvector, (size_t)S.sizeV, kSlotIO + 9, &dV);
    if (rc == NRG_OK) {
        const int nbo = io->numberOfBasis_old;
        const std::vector<HostSeg> segs = spike_ims_segs(M, it, cfs ? nullptr : &gs, nbo);
        rc = stage_in_segs(ctx, io->invariant_matrix_spectrum, (size_t)nbo * nbo * M.nMat, nbo, segs,
                           kSlotIO + 10, &dIMS);
    }
    if (rc == NRG_OK && cfs) {
        // only the density blocks of this iteration's sectors are staged (one contiguous
        // range of the caller's array); offsets become relative to the range
        long long lo = -1, hi = -1;
        for (int s = 0; s < S.nsub; ++s) {
            if (it.rdm_off[s] < 0) continue;
            const long long a = it.rdm_off[s], b = a + (long long)it.kept[s] * it.kept[s];
            lo = lo < 0 ? a : std::min(lo, a);
            hi = std::max(hi, b);
        }
        if (lo >= 0) {
            if (hi > (long long)io->sizeOfReducedDensity) {
                nrg_set_error_message("reduced density blocks beyond sizeOfReducedDensity");
                rc = NRG_ERR_INVALID;
            } else {
                rc = stage_in(ctx, io->reducedDensityMatrix + lo, (size_t)(hi - lo), kSlotIO + 11, &dR);
                for (int s = 0; s < S.nsub; ++s)
                    if (it.rdm_off[s] >= 0) it.rdm_off[s] -= lo;
            }
        }
    }
    DevBuf& bE = ctx->slot(kSlotIO + 12);
    if (rc == NRG_OK) rc = bE.ensure(sizeof(double) * std::max(nbf, 1));
    if (rc == NRG_OK && cudaMemcpyAsync(bE.p, Esec.data(), sizeof(double) * nbf, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess) rc = NRG_ERR_CUDA;
    dEs = bE.as<double>();
    it.d_V = dV; it.d_Esec = dEs; it.d_rdm = dR; it.nb_kept = io->numberOfBasis;
    // per-iteration bins (tmpBinnedSpike*, :304-325), zeroed
    const size_t nw = (size_t)nbin * M.nMat;
    DevBuf& tb = ctx->slot(kSlotIO + 13);
    DevBuf& tt = ctx->slot(kSlotIO + 14);
    if (rc == NRG_OK) rc = tb.ensure(sizeof(double) * 2 * nw);
    if (rc == NRG_OK) rc = tt.ensure(sizeof(double) * 4 * M.nMat);
    double* tPos = tb.as<double>();
    double* tNeg = tPos + nw;
    double* tot = tt.as<double>();
    if (rc == NRG_OK) rc = run_fill(ctx, tPos, (long long)(2 * nw), 0.0);
    if (rc == NRG_OK) rc = run_fill(ctx, tot, 4LL * M.nMat, 0.0);
    clk.mark(0);
    if (rc == NRG_OK) {
        OpView old;
        old.dense = dIMS;
        old.nb = io->numberOfBasis_old;
        if (cfs) rc = spike_cfs_device(ctx, iteration, it, old, dR, tPos, tNeg, tot);
        else rc = spike_t0_device(ctx, iteration, it, gs, old, tPos, tNeg);
    }
    clk.mark(1);
    // add into the caller's bins (weight column = second column)
    std::vector<double> hp(nw), hn(nw);
    if (rc == NRG_OK && cudaMemcpyAsync(hp.data(), tPos, sizeof(double) * nw, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess) rc = NRG_ERR_CUDA;
    if (rc == NRG_OK && cudaMemcpyAsync(hn.data(), tNeg, sizeof(double) * nw, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess) rc = NRG_ERR_CUDA;
    std::vector<double> htot(4 * M.nMat, 0.0);
    if (rc == NRG_OK && cudaMemcpyAsync(htot.data(), tot, sizeof(double) * 2 * M.nMat, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess) rc = NRG_ERR_CUDA;
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess && rc == NRG_OK) rc = NRG_ERR_CUDA;
    if (rc == NRG_OK) rc = check_device_status(ctx);
    if (rc == NRG_OK) {
        const bool dev_bins = is_device_ptr(io->binnedSpikePositive);
        std::vector<double> bp, bn;
        double *wp, *wn;
        if (dev_bins) {
            bp.resize(nw); bn.resize(nw);
            cudaMemcpy(bp.data(), io->binnedSpikePositive + nw, sizeof(double) * nw, cudaMemcpyDeviceToHost);
            cudaMemcpy(bn.data(), io->binnedSpikeNegative + nw, sizeof(double) * nw, cudaMemcpyDeviceToHost);
            wp = bp.data(); wn = bn.data();
        } else {
            wp = io->binnedSpikePositive + nw;
            wn = io->binnedSpikeNegative + nw;
        }
        for (int m = 0; m < M.nMat; ++m) {
            double sp = 0.0, sn = 0.0;
            for (int i = 0; i < nbin; ++i) { sp += hp[(size_t)m * nbin + i]; sn += hn[(size_t)m * nbin + i]; }
            htot[2 * M.nMat + 2 * m] = sn;
            htot[2 * M.nMat + 2 * m + 1] = sp;
        }
        for (size_t i = 0; i < nw; ++i) { wp[i] += hp[i]; wn[i] += hn[i]; }
        if (dev_bins) {
            cudaMemcpy(io->binnedSpikePositive + nw, bp.data(), sizeof(double) * nw, cudaMemcpyHostToDevice);
            cudaMemcpy(io->binnedSpikeNegative + nw, bn.data(), sizeof(double) * nw, cudaMemcpyHostToDevice);
        }
        if (io->total_sum) {
            // [raw negative, raw positive, binned negative, binned positive] per matrix
            for (int m = 0; m < M.nMat; ++m) {
                io->total_sum[4 * m + 0] = htot[2 * m + 0];
                io->total_sum[4 * m + 1] = htot[2 * m + 1];
                io->total_sum[4 * m + 2] = htot[2 * M.nMat + 2 * m];
                io->total_sum[4 * m + 3] = htot[2 * M.nMat + 2 * m + 1];
            }
        }
    }
    swap_tables(ctx, S, 0);
    clk.mark(2);
    return rc;
}

int nrg_broaden_log_gaussian(nrg_context* ctx, const double* bins, int32_t numberOfBin, int32_t nMat, double b,
                             const double* omega, int32_t nOmega, double* A) {
    if (!ctx) { nrg_set_error_message("NULL context"); return NRG_ERR_INVALID; }
    if (numberOfBin < 1 || nMat < 1 || nOmega < 0 || !(b > 0.0)) {
        nrg_set_error_message("nrg_broaden_log_gaussian: numberOfBin %d, nMat %d, nOmega %d, b %g", numberOfBin, nMat,
                              nOmega, b);
        return NRG_ERR_INVALID;
    }
    if (nOmega == 0) return NRG_OK;
    NRG_CUDA_TRY(cudaSetDevice(ctx->device));
    NRG_TRY(reject_foreign(ctx, "nrg_broaden_log_gaussian", {bins, omega, A}));
    const double *dB = nullptr, *dW = nullptr;
    double* dA = nullptr;
    const size_t nbt = 2 * (size_t)numberOfBin * nMat;
    NRG_TRY(stage_in(ctx, bins, nbt, kSlotIO + 15, &dB));
    NRG_TRY(stage_in(ctx, omega, (size_t)nOmega, kSlotIO + 16, &dW));
    NRG_TRY(stage_out(ctx, A, (size_t)nOmega * nMat, kSlotIO + 17, &dA));
    NRG_TRY(run_broaden(ctx, dB, numberOfBin, nMat, b, dW, nOmega, dA));
    NRG_TRY(finish_out(ctx, A, dA, (size_t)nOmega * nMat));
    NRG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return NRG_OK;
}

int nrg_spike_zero_temperature(nrg_context* ctx, int32_t iteration, const nrg_spike_io* io) {
    return spike_common(ctx, iteration, io, false);
}
int nrg_spike_cfs(nrg_context* ctx, int32_t iteration, const nrg_spike_io* io) {
    return spike_common(ctx, iteration, io, true);
}

}  // extern "C"
