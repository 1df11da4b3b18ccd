// Device-side implementations of the reference routines, shared by the C ABI (capi.cu)
// and the device-resident driver (driver.cu).
#include "internal.hpp"

#include <map>
#include <mutex>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <unordered_set>

namespace nrg {

// ------------------------------------------------------------------------------------
// DevBuf
// ------------------------------------------------------------------------------------
int DevBuf::ensure(size_t want) {
    if (want <= bytes && p) return NRG_OK;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    size_t sz = want < 256 ? 256 : want;
    sz = (sz + 255) & ~size_t(255);
    cudaError_t e = cudaMalloc(&p, sz);
    if (e != cudaSuccess) {
        p = nullptr;
        nrg_set_error_message("cudaMalloc(%zu) failed: %s", sz, cudaGetErrorString(e));
        return NRG_ERR_NOMEM;
    }
    bytes = sz;
    return NRG_OK;
}
void DevBuf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
}

int HostBuf::ensure(size_t want, bool keep) {
    if (want <= bytes && p && alloc_pageable == pageable) return NRG_OK;
    size_t sz = want < 4096 ? 4096 : want;
    if (keep) sz = std::max(sz, bytes + bytes / 2);
    sz = (sz + 4095) & ~size_t(4095);
    void* q = nullptr;
    if (pageable) {
        q = std::malloc(sz);
        if (!q) {
            nrg_set_error_message("malloc(%zu) failed", sz);
            return NRG_ERR_NOMEM;
        }
    } else {
        cudaError_t e = cudaHostAlloc(&q, sz, cudaHostAllocPortable);
        if (e != cudaSuccess) {
            nrg_set_error_message("cudaHostAlloc(%zu) failed: %s", sz, cudaGetErrorString(e));
            return NRG_ERR_NOMEM;
        }
    }
    if (keep && p && bytes) std::memcpy(q, p, std::min(bytes, sz));
    release();
    p = q;
    bytes = sz;
    alloc_pageable = pageable;
    return NRG_OK;
}
void HostBuf::release() {
    if (p) {
        if (alloc_pageable) std::free(p);
        else cudaFreeHost(p);
    }
    p = nullptr;
    bytes = 0;
}

// ------------------------------------------------------------------------------------
// Model
// ------------------------------------------------------------------------------------
double Model::scale(int N) const {
    // module.F90:690-711
    if (scalingType == 0) return std::pow(Lambda, -double(N) * 0.5);
    if (scalingType == 1)
        return D * 0.5 * (1.0 + 1.0 / Lambda) * std::pow(Lambda, -double(N) * 0.5 - z + 1.0);
    return std::pow(Lambda, -double(N) * 0.5 - z) * D * (Lambda - 1.0) / std::log(Lambda);
}
int Model::numberOfBin() const {
    // main.F90:142-144
    const double Emax = scale(-1);
    const double log10Emax = double((int)std::log10(Emax)) + 1.0;
    return (int)(log10Emax - (-15.0)) * 1000 + 1;
}

// ------------------------------------------------------------------------------------
// Sectors
// ------------------------------------------------------------------------------------
int Sectors::build(int nsub_, const int* si, int nb_, const int* bi, int nVar_, int nOps_) {
    nsub = nsub_; nb = nb_; nVar = nVar_; nOps = nOps_;
    const int rs = nVar + 3;
    qnHash.clear();   // rebuilt below once the table is valid
    qn.assign((size_t)nsub * nVar, 0);
    dim.assign(nsub, 0);
    start.assign(nsub, 0);
    ce.assign(nsub, 0);
    long long acc = 0;
    for (int s = 0; s < nsub; ++s) {
        for (int v = 0; v < nVar; ++v) qn[(size_t)s * nVar + v] = si[(size_t)s * rs + v];
        dim[s] = si[(size_t)s * rs + nVar];
        start[s] = si[(size_t)s * rs + nVar + 2] - 1;
        ce[s] = acc;
        const long long ref_ce = (long long)si[(size_t)s * rs + nVar + 1] - 1;
        if (acc < 0x7fffffffLL && ref_ce != acc) {
            nrg_set_error_message("subspaceInfo(%d)%%count_eigenvector=%lld, expected %lld", s + 1,
                                  ref_ce + 1, acc + 1);
            return NRG_ERR_INVALID;
        }
        if (dim[s] < 1 || start[s] < 0 || start[s] + dim[s] > nb) {
            nrg_set_error_message("subspaceInfo(%d) out of range", s + 1);
            return NRG_ERR_INVALID;
        }
        acc += (long long)dim[s] * dim[s];
    }
    sizeV = acc;
    index_qn();
    rowOp.resize(nb); rowRef.resize(nb); rowVar.resize(nb);
    for (int i = 0; i < nb; ++i) {
        rowRef[i] = bi[(size_t)i * rs + nVar] - 1;
        rowVar[i] = bi[(size_t)i * rs + nVar + 1];
        rowOp[i] = bi[(size_t)i * rs + nVar + 2] - 1;
        if (rowOp[i] < 0 || rowOp[i] >= nOps) {
            nrg_set_error_message("basis_input(%d)%%operation out of range", i + 1);
            return NRG_ERR_INVALID;
        }
    }
    // rows per (sector, operation), in row order
    lstOff.assign((size_t)nsub * nOps + 1, 0);
    for (int s = 0; s < nsub; ++s)
        for (int i = start[s]; i < start[s] + dim[s]; ++i) lstOff[(size_t)s * nOps + rowOp[i] + 1]++;
    for (size_t x = 1; x < lstOff.size(); ++x) lstOff[x] += lstOff[x - 1];
    lst.assign(lstOff.back(), 0);
    std::vector<int> fill(lstOff.begin(), lstOff.end() - 1);
    for (int s = 0; s < nsub; ++s)
        for (int i = start[s]; i < start[s] + dim[s]; ++i)
            lst[fill[(size_t)s * nOps + rowOp[i]]++] = i - start[s];
    // the rows of one (sector, operation) descend from one previous sector: they must list
    // its states by column 1, 2, ... with consecutive references
    refBase.assign((size_t)nsub * nOps, -1);
    for (int s = 0; s < nsub; ++s) {
        for (int a = 0; a < nOps; ++a) {
            const int o0 = lstOff[(size_t)s * nOps + a], o1 = lstOff[(size_t)s * nOps + a + 1];
            if (o1 == o0) continue;
            const int r0 = rowRef[start[s] + lst[o0]];
            refBase[(size_t)s * nOps + a] = r0;
            for (int q = o0; q < o1; ++q) {
                const int row = start[s] + lst[q];
                if (rowVar[row] != q - o0 + 1 || rowRef[row] != r0 + (q - o0)) {
                    nrg_set_error_message(
                        "sector %d operation %d: rows are not the previous sector's states in "
                        "column order (variation %d, reference %d)", s + 1, a + 1, rowVar[row],
                        rowRef[row] + 1);
                    return NRG_ERR_UNSUPPORTED;
                }
            }
        }
    }
    return NRG_OK;
}

int Sectors::upload(nrg_context* ctx) {
    const int rs = nVar + 3;
    std::vector<int> bi((size_t)nb * rs, 0);
    for (int i = 0; i < nb; ++i) {
        bi[(size_t)i * rs + nVar] = rowRef[i] + 1;
        bi[(size_t)i * rs + nVar + 1] = rowVar[i];
        bi[(size_t)i * rs + nVar + 2] = rowOp[i] + 1;
    }
    NRG_TRY(d_bi.ensure(sizeof(int) * bi.size()));
    NRG_TRY(d_lst.ensure(sizeof(int) * (lst.size() + 1)));
    NRG_TRY(d_lstOff.ensure(sizeof(int) * lstOff.size()));
    NRG_TRY(h2d_async(ctx, d_bi.p, bi.data(), sizeof(int) * bi.size()));
    NRG_TRY(h2d_async(ctx, d_lst.p, lst.data(), sizeof(int) * lst.size()));
    NRG_TRY(h2d_async(ctx, d_lstOff.p, lstOff.data(), sizeof(int) * lstOff.size()));
    return NRG_OK;
}

int raise_smem_limit(const void* func, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, size_t> limit;
    int dev = 0;
    NRG_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    size_t& cur = limit[{func, dev}];
    if (bytes > cur) {
        NRG_CUDA_TRY(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
        cur = bytes;
    }
    return NRG_OK;
}

int h2d_async(nrg_context* ctx, void* dst, const void* src, size_t bytes) {
    if (bytes == 0) return NRG_OK;
    ctx->h2d += (long long)bytes;
    const size_t need = (bytes + 255) & ~size_t(255);
    if (!ctx->stage_host) {
        const size_t cap = size_t(64) << 20;
        void* p = nullptr;
        NRG_CUDA_TRY(cudaHostAlloc(&p, cap, cudaHostAllocDefault));
        ctx->stage_host = static_cast<char*>(p);
        ctx->stage_cap = cap;
        ctx->stage_head = 0;
    }
    if (need > ctx->stage_cap / 2) {   // large: plain copy (waits for the stream)
        NRG_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
        return NRG_OK;
    }
    size_t begin = ctx->stage_head;
    if (begin + need > ctx->stage_cap) begin = 0;
    const size_t end = begin + need;
    auto& fl = ctx->stage_inflight;
    while (!fl.empty() && cudaEventQuery(fl.front().ev) == cudaSuccess) {
        ctx->event_pool.push_back(fl.front().ev);
        fl.pop_front();
    }
    for (auto& c : fl)
        if (c.begin < end && begin < c.end) NRG_CUDA_TRY(cudaEventSynchronize(c.ev));
    std::memcpy(ctx->stage_host + begin, src, bytes);
    NRG_CUDA_TRY(cudaMemcpyAsync(dst, ctx->stage_host + begin, bytes, cudaMemcpyHostToDevice, ctx->stream));
    cudaEvent_t ev;
    if (!ctx->event_pool.empty()) {
        ev = ctx->event_pool.back();
        ctx->event_pool.pop_back();
    } else {
        NRG_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    }
    NRG_CUDA_TRY(cudaEventRecord(ev, ctx->stream));
    fl.push_back({begin, end, ev});
    ctx->stage_head = end;
    return NRG_OK;
}

// index by quantum numbers: the first sector of each qn (findSubspace semantics)
void Sectors::index_qn() {
    size_t cap = 16;
    while (cap < 4 * (size_t)nsub) cap <<= 1;
    qnHash.assign(cap, -1);
    for (int s = 0; s < nsub; ++s) {
        const int* q = &qn[(size_t)s * nVar];
        for (size_t x = hash_qn(q, nVar) & (cap - 1);; x = (x + 1) & (cap - 1)) {
            const int o = qnHash[x];
            if (o < 0) { qnHash[x] = s; break; }
            bool eq = true;
            for (int v = 0; v < nVar; ++v)
                if (qn[(size_t)o * nVar + v] != q[v]) { eq = false; break; }
            if (eq) break;   // an earlier sector has these qn: it stays the one found
        }
    }
}

unsigned long long Sectors::hash_qn(const int* q, int nVar) {
    unsigned long long h = 1469598103934665603ULL;   // FNV-1a over the quantum numbers
    for (int v = 0; v < nVar; ++v) {
        h ^= (unsigned long long)(unsigned)q[v];
        h *= 1099511628211ULL;
    }
    return h;
}

int Sectors::find(const int* q) const {
    if (qnHash.empty()) {
        for (int s = 0; s < nsub; ++s) {
            bool eq = true;
            for (int v = 0; v < nVar; ++v)
                if (qn[(size_t)s * nVar + v] != q[v]) { eq = false; break; }
            if (eq) return s;
        }
        return -1;
    }
    const size_t mask = qnHash.size() - 1;
    for (size_t x = hash_qn(q, nVar) & mask;; x = (x + 1) & mask) {
        const int s = qnHash[x];
        if (s < 0) return -1;
        bool eq = true;
        for (int v = 0; v < nVar; ++v)
            if (qn[(size_t)s * nVar + v] != q[v]) { eq = false; break; }
        if (eq) return s;
    }
}

int check_device_status(nrg_context* ctx) {
    int st = 0;
    NRG_CUDA_TRY(cudaMemcpyAsync(&st, ctx->d_status.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    NRG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (st != 0) {
        NRG_CUDA_TRY(cudaMemsetAsync(ctx->d_status.p, 0, sizeof(int), ctx->stream));
        nrg_set_error_message("device status flags 0x%x (1: index out of range, 4: secular root, 8: NaN or Inf "
                              "in a block)", st);
        return (st & (NRG_DEV_SECULAR | NRG_DEV_NONFINITE)) ? NRG_ERR_NUMERIC : NRG_ERR_INVALID;
    }
    return NRG_OK;
}

// ------------------------------------------------------------------------------------
// diagonalization (diagonalization.F90:1-410)
// ------------------------------------------------------------------------------------
int diag_device(nrg_context* ctx, int iteration, Sectors& S, const double* d_Eold, int nb_old,
                const double* d_IMold, double* d_V, double* d_E, DiagOut* out, DiagPost* post) {
    const bool early = post && post->early;
    double* h_E = post ? post->h_E : nullptr;
    TruncTables* trunc = post ? post->trunc : nullptr;
    const int nsec = S.nsub;
    std::vector<int> order(nsec);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return S.dim[a] > S.dim[b]; });
    std::vector<SyevSector> secs(nsec);
    std::vector<long long> colPrefix(nsec);
    std::vector<int> secStart(nsec);
    long long wsd = 0, wsi = 0, cols = 0;
    int max_n = 1, nlarge = 0;
    std::vector<SyevSector> large;
    for (int x = 0; x < nsec; ++x) {
        const int s = order[x];
        SyevSector& q = secs[x];
        q.n = S.dim[s];
        q.a_off = S.ce[s];
        q.e_off = S.start[s];
        q.w_off = 0;
        q.i_off = 0;
        q.pad = 0;
        if (q.n > kLargeSector) {
            large.push_back(q);
            ++nlarge;
        } else {
            q.w_off = wsd;
            q.i_off = wsi;
            wsd += syev_ws_doubles(q.n);
            wsi += syev_ws_ints(q.n);
            max_n = std::max(max_n, q.n);
        }
        colPrefix[x] = cols;
        cols += q.n;
        secStart[x] = S.start[s];
    }
    DevBuf& bsec = ctx->scratch.b[0];
    DevBuf& bcol = ctx->scratch.b[1];
    DevBuf& bstart = ctx->scratch.b[2];
    DevBuf& bwd = ctx->scratch.b[3];
    DevBuf& bwi = ctx->scratch.b[4];
    DevBuf& bmin = ctx->scratch.b[5];
    NRG_TRY(bsec.ensure(sizeof(SyevSector) * nsec));
    NRG_TRY(bcol.ensure(sizeof(long long) * nsec));
    NRG_TRY(bstart.ensure(sizeof(int) * nsec));
    NRG_TRY(bwd.ensure(sizeof(double) * (size_t)std::max(wsd, 1LL)));
    NRG_TRY(bwi.ensure(sizeof(int) * (size_t)std::max(wsi, 1LL)));
    NRG_TRY(bmin.ensure(sizeof(double) * 2));
    NRG_TRY(h2d_async(ctx, bsec.p, secs.data(), sizeof(SyevSector) * nsec));
    NRG_TRY(h2d_async(ctx, bcol.p, colPrefix.data(), sizeof(long long) * nsec));
    NRG_TRY(h2d_async(ctx, bstart.p, secStart.data(), sizeof(int) * nsec));
    NRG_TRY(run_assemble(ctx, iteration, S, bsec.as<SyevSector>(), bcol.as<long long>(), bstart.as<int>(),
                         nsec, cols, d_Eold, nb_old, d_IMold, d_V));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (ctx->profiling) {
        NRG_CUDA_TRY(cudaEventCreate(&e0));
        NRG_CUDA_TRY(cudaEventCreate(&e1));
        NRG_CUDA_TRY(cudaEventRecord(e0, ctx->stream));
    }
    // Three independent groups: the largest large sectors (order >= 4/5 of the largest)
    // on a stream of the greatest priority, the other sectors of order > 128 on a third
    // stream, and the sectors of order <= 128 (one block each) on the second stream.  The
    // largest sectors' pipeline sets the critical path; the blocks of the other groups
    // fill the SMs it leaves idle.
    // With early eigenvalues the largest sectors always take their own stream, so that
    // the caller's stream can pick up the eigenvalues before the back-transformations
    // end; without a second large group that stream has the normal priority (the
    // priority only orders the two large groups of one instance, and independent
    // instances side by side should not all claim the greatest one).
    std::vector<SyevSector> g1, g2;
    for (const auto& q : large) (5 * q.n >= 4 * large[0].n ? g1 : g2).push_back(q);
    const bool fork_small = nsec > nlarge && nlarge > 0;
    const bool fork_large = !g2.empty() || (early && !g1.empty());
    cudaStream_t s1 = nullptr;
    if (!ctx->aux) {
        int lo = 0, hi = 0;
        NRG_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&lo, &hi));
        NRG_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->aux, cudaStreamNonBlocking));
        NRG_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->aux2, cudaStreamNonBlocking));
        NRG_CUDA_TRY(cudaStreamCreateWithPriority(&ctx->aux_hi, cudaStreamNonBlocking, hi));
        for (cudaEvent_t* e : {&ctx->ev_fork, &ctx->ev_join, &ctx->ev_join2, &ctx->ev_join_hi, &ctx->ev_evals_hi,
                               &ctx->ev_evals2, &ctx->ev_evals_host})
            NRG_CUDA_TRY(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    }
    if (fork_small || fork_large) NRG_CUDA_TRY(cudaEventRecord(ctx->ev_fork, ctx->stream));
    int rl = NRG_OK;
    if (fork_large) {
        s1 = g2.empty() ? ctx->aux2 : ctx->aux_hi;
        NRG_CUDA_TRY(cudaStreamWaitEvent(s1, ctx->ev_fork, 0));
        cudaStream_t caller = ctx->stream;
        ctx->stream = s1;
        rl = syev_large(ctx, g1, d_V, d_E, 24, early && !g1.empty() ? ctx->ev_evals_hi : nullptr);
        ctx->stream = caller;
        NRG_CUDA_TRY(cudaEventRecord(ctx->ev_join_hi, s1));
    } else {
        rl = syev_large(ctx, g1, d_V, d_E, 24);
    }
    if (fork_small) NRG_CUDA_TRY(cudaStreamWaitEvent(ctx->aux, ctx->ev_fork, 0));
    if (nsec > nlarge && rl == NRG_OK) {
        rl = launch_syev(bsec.as<SyevSector>() + nlarge, nsec - nlarge, max_n, d_V, d_E, bwd.as<double>(),
                         bwi.as<int>(), ctx->d_status.as<int>(), fork_small ? ctx->aux : ctx->stream);
        ctx->launches++;
    }
    if (fork_small) NRG_CUDA_TRY(cudaEventRecord(ctx->ev_join, ctx->aux));
    const bool has_g2 = fork_large && !g2.empty();
    if (has_g2) {
        NRG_CUDA_TRY(cudaStreamWaitEvent(ctx->aux2, ctx->ev_fork, 0));
        cudaStream_t caller = ctx->stream;
        ctx->stream = ctx->aux2;
        if (rl == NRG_OK) rl = syev_large(ctx, g2, d_V, d_E, 31, early ? ctx->ev_evals2 : nullptr);
        ctx->stream = caller;
        NRG_CUDA_TRY(cudaEventRecord(ctx->ev_join2, ctx->aux2));
    }
    NRG_TRY(rl);
    // The drop-in's eigenvectors to the caller's page-locked array as their groups end: the
    // blocks outside the largest class once the small sectors and the second large group are
    // done (while the largest sectors are still being reduced), the largest class's after
    // it; each part chopped (diagonalization.F90:273-280) just before its copy.
    const bool copy_early = !early && post && post->h_V && !g1.empty() && (fork_small || has_g2);
    if (copy_early) {
        if (!ctx->aux_copy) {
            NRG_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->aux_copy, cudaStreamNonBlocking));
            NRG_CUDA_TRY(cudaEventCreateWithFlags(&ctx->ev_copied, cudaEventDisableTiming));
        }
        cudaStream_t cs = ctx->aux_copy;
        if (!fork_large) NRG_CUDA_TRY(cudaEventRecord(ctx->ev_join_hi, ctx->stream));   // g1 ran there
        std::vector<std::pair<long long, long long>> hi, rest;   // (offset, length) in doubles
        for (const auto& q : g1) hi.push_back({q.a_off, (long long)q.n * q.n});
        std::sort(hi.begin(), hi.end());
        long long pos = 0;
        for (const auto& r : hi) {
            if (r.first > pos) rest.push_back({pos, r.first - pos});
            pos = r.first + r.second;
        }
        if (pos < S.sizeV) rest.push_back({pos, S.sizeV - pos});
        auto chop_copy = [&](const std::vector<std::pair<long long, long long>>& parts) -> int {
            for (const auto& r : parts) {
                NRG_TRY(run_eig_chop(ctx, r.second, d_V + r.first, cs));
                NRG_CUDA_TRY(cudaMemcpyAsync(post->h_V + r.first, d_V + r.first, sizeof(double) * r.second,
                                             cudaMemcpyDeviceToHost, cs));
                ctx->d2h += (long long)sizeof(double) * r.second;
            }
            return NRG_OK;
        };
        if (fork_small) NRG_CUDA_TRY(cudaStreamWaitEvent(cs, ctx->ev_join, 0));
        if (has_g2) NRG_CUDA_TRY(cudaStreamWaitEvent(cs, ctx->ev_join2, 0));
        NRG_TRY(chop_copy(rest));
        NRG_CUDA_TRY(cudaStreamWaitEvent(cs, ctx->ev_join_hi, 0));
        NRG_TRY(chop_copy(hi));
        NRG_CUDA_TRY(cudaEventRecord(ctx->ev_copied, cs));
        NRG_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, ctx->ev_copied, 0));
        post->copied_V = true;
    }
    double* hs = nullptr;
    if (early) {
        // eigenvalues of every group -> shift -> host, then the eigenvectors' join
        NRG_TRY(ctx->h_small.ensure(64));
        hs = ctx->h_small.as<double>();
        if (fork_large && !g1.empty()) NRG_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, ctx->ev_evals_hi, 0));
        if (has_g2) NRG_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, ctx->ev_evals2, 0));
        if (fork_small) NRG_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, ctx->ev_join, 0));
        NRG_TRY(run_eig_shift(ctx, d_E, S.nb, bmin.as<double>()));
        if (trunc) NRG_TRY(trunc->launch(ctx, d_E));
        if (h_E) {
            NRG_CUDA_TRY(cudaMemcpyAsync(h_E, d_E, sizeof(double) * S.nb, cudaMemcpyDeviceToHost, ctx->stream));
            ctx->d2h += (long long)sizeof(double) * S.nb;
        }
        NRG_CUDA_TRY(cudaMemcpyAsync(hs, bmin.p, sizeof(double) * 2, cudaMemcpyDeviceToHost, ctx->stream));
        NRG_CUDA_TRY(cudaMemcpyAsync(hs + 2, ctx->d_status.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        ctx->d2h += (long long)sizeof(double) * 2 + (long long)sizeof(int);
        NRG_CUDA_TRY(cudaEventRecord(ctx->ev_evals_host, ctx->stream));
    }
    if (fork_large) NRG_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, ctx->ev_join_hi, 0));
    if (has_g2) NRG_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, ctx->ev_join2, 0));
    if (fork_small && !early) NRG_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, ctx->ev_join, 0));
    if (ctx->profiling) {
        NRG_CUDA_TRY(cudaEventRecord(e1, ctx->stream));
        double f = 0.0;
        for (int s = 0; s < nsec; ++s) f += (4.0 / 3.0 + 2.0) * double(S.dim[s]) * S.dim[s] * S.dim[s];
        ctx->pending_syev.push_back({e0, e1, f, 0.0});
        if (!early) NRG_TRY(flush_profile_timers(ctx));
    }
    if (early) {
        NRG_TRY(run_eig_chop(ctx, S.sizeV, d_V));
        NRG_CUDA_TRY(cudaEventSynchronize(ctx->ev_evals_host));
        if (out) {
            out->groundStateEnergy = hs[1];
            out->emin = hs[0];
        }
        int st = 0;
        std::memcpy(&st, hs + 2, sizeof(int));
        if (st != 0) return check_device_status(ctx);   // reports and clears the flags
        return NRG_OK;
    }
    NRG_TRY(run_eig_shift(ctx, d_E, S.nb, bmin.as<double>()));
    if (trunc) NRG_TRY(trunc->launch(ctx, d_E));
    if (!copy_early) NRG_TRY(run_eig_chop(ctx, S.sizeV, d_V));
    double mg[2];
    NRG_CUDA_TRY(cudaMemcpyAsync(mg, bmin.p, sizeof(double) * 2, cudaMemcpyDeviceToHost, ctx->stream));
    ctx->d2h += sizeof(mg);
    NRG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (out) {
        out->groundStateEnergy = mg[1];
        out->emin = mg[0];
    }
    return check_device_status(ctx);
}

int flush_profile_timers(nrg_context* ctx) {
    for (auto& t : ctx->pending_syev) {
        float ms = 0.f;
        NRG_CUDA_TRY(cudaEventSynchronize(t.b));
        NRG_CUDA_TRY(cudaEventElapsedTime(&ms, t.a, t.b));
        cudaEventDestroy(t.a);
        cudaEventDestroy(t.b);
        ctx->syev_ms += ms;
        ctx->syev_launches++;
        ctx->syev_flops += t.flops;
    }
    ctx->pending_syev.clear();
    for (auto& t : ctx->pending_tri) {
        float tm = 0.f;
        NRG_CUDA_TRY(cudaEventSynchronize(t.b));
        NRG_CUDA_TRY(cudaEventElapsedTime(&tm, t.a, t.b));
        cudaEventDestroy(t.a);
        cudaEventDestroy(t.b);
        ctx->tri_launches++;
        ctx->tri_ms += tm;
        ctx->tri_flops += t.flops;
        ctx->tri_bytes += t.bytes;
    }
    ctx->pending_tri.clear();
    return NRG_OK;
}

std::vector<int> kept_per_sector(const Sectors& S, int nb_kept, const int* bo) {
    // invariantMatrixDGEMM.F90:84-100: count kept states whose quantum numbers match
    std::vector<int> kept(S.nsub, 0);
    const int rs = S.nVar + 3;
    for (int i = 0; i < nb_kept; ++i) {
        const int s = S.find(bo + (size_t)i * rs);
        if (s >= 0) kept[s]++;
    }
    return kept;
}

// ------------------------------------------------------------------------------------
// invariant matrices
// ------------------------------------------------------------------------------------
int invmat_device(nrg_context* ctx, const Sectors& S, const std::vector<int>& kept,
                  const double* d_V, double* d_IM) {
    // invariantMatrixDGEMM.F90:67-341
    const Model& M = ctx->model;
    const int nsub = S.nsub, nVar = S.nVar;
    std::vector<long long> kst(nsub + 1, 0);
    for (int s = 0; s < nsub; ++s) kst[s + 1] = kst[s] + kept[s];
    const long long nbk = kst[nsub];
    NRG_TRY(run_fill(ctx, d_IM, nbk * nbk * M.nCM, 0.0));
    const int cs = M.cb[0], ce_ = M.cb[2], ss = M.cb[1], se = M.cb[3];
    std::vector<ImGatherProb> gp;
    long long toff = 0;
    for (int L = 0; L < nsub; ++L) {
        if (kept[L] == 0) continue;
        for (int R = 0; R < nsub; ++R) {
            if (kept[R] == 0) continue;
            int dQ = 0, dS = 0;
            for (int v = ss; v <= se; ++v) dS += S.qn[(size_t)L * nVar + v - 1] - S.qn[(size_t)R * nVar + v - 1];
            if (cs == ce_ && cs == 0) {
                if (std::abs(dS) != 1) continue;
            } else {
                for (int v = cs; v <= ce_; ++v) dQ += S.qn[(size_t)L * nVar + v - 1] - S.qn[(size_t)R * nVar + v - 1];
                if (dQ != 1 || std::abs(dS) != 1) continue;
            }
            for (int t = 0; t < M.nCM; ++t) {
                ImGatherProb p;
                p.t_off = toff; p.vR_off = S.ce[R]; p.L = L; p.R = R; p.t = t;
                p.dL = S.dim[L]; p.dR = S.dim[R]; p.kR = kept[R]; p.startL = S.start[L];
                gp.push_back(p);
                toff += (long long)p.dL * p.kR;
            }
        }
    }
    if (gp.empty()) return NRG_OK;
    DevBuf& T = ctx->scratch.b[6];
    NRG_TRY(T.ensure(sizeof(double) * (size_t)toff));
    NRG_TRY(run_im_gather(ctx, S, gp, d_V, T.as<double>()));
    std::vector<GemmProblem> probs;
    for (const auto& g : gp) {
        GemmProblem P;
        std::memset(&P, 0, sizeof(P));
        P.M = kept[g.L]; P.N = kept[g.R]; P.K = g.dL;
        P.alpha = 1.0; P.beta = 0.0;
        P.A = d_V + S.ce[g.L]; P.a_si = g.dL; P.a_sk = 1;
        P.B = T.as<double>() + g.t_off; P.b_sk = 1; P.b_sj = g.dL;
        P.C = d_IM + kst[g.R] + kst[g.L] * nbk + (long long)g.t * nbk * nbk;
        P.c_si = nbk; P.c_sj = 1;
        probs.push_back(P);
    }
    return launch_ggemm(ctx, probs, 8);
}

int SparseBlocks::sector_of(long long i) const {
    if (i < 0 || nsub == 0 || i >= kst[nsub]) return -1;
    const int s = (int)(std::upper_bound(kst.begin(), kst.end(), i) - kst.begin()) - 1;
    return (s >= 0 && s < nsub && kept[s] > 0) ? s : -1;
}

const double* OpView::at(long long r0, long long l0, int m, long long cr, long long cl, long long* sr,
                         long long* sl, bool* bad) const {
    *bad = false;
    if (dense) {
        if (r0 < 0 || l0 < 0 || r0 + cr > nb || l0 + cl > nb) { *bad = true; return nullptr; }
        *sr = 1;
        *sl = nb;
        return dense + r0 + l0 * nb + (long long)m * nb * nb;
    }
    if (!sp) { *bad = true; return nullptr; }
    const int R = sp->sector_of(r0), L = sp->sector_of(l0);
    if (R < 0 || L < 0 || r0 + cr > sp->kst[R] + sp->kept[R] || l0 + cl > sp->kst[L] + sp->kept[L]) {
        *bad = true;
        return nullptr;
    }
    const long long o = sp->off[((size_t)L * sp->nsub + R) * sp->nMat + m];
    if (o < 0) return nullptr;
    *sr = 1;
    *sl = sp->kept[R];
    return sp->data + o + (r0 - sp->kst[R]) + (l0 - sp->kst[L]) * sp->kept[R];
}

int invmat_spec_device(nrg_context* ctx, const Sectors& S, const std::vector<int>& kept,
                       const double* d_V, const OpView& old, double* d_dense, SparseBlocks* sp_out,
                       DevBuf* sp_buf) {
    // invariantMatrixForSpectrumDGEMM.F90:71-370
    const Model& M = ctx->model;
    const int nsub = S.nsub, nVar = S.nVar, nOps = S.nOps;
    std::vector<long long> kst(nsub + 1, 0);
    for (int s = 0; s < nsub; ++s) kst[s + 1] = kst[s] + kept[s];
    const long long nbk = kst[nsub];
    if (d_dense) NRG_TRY(run_fill(ctx, d_dense, nbk * nbk * M.nMat, 0.0));
    struct Pair { int L, R, m; long long t_off; };
    std::vector<Pair> pairs;
    long long toff = 0;
    for (int L = 0; L < nsub; ++L) {
        if (kept[L] == 0) continue;
        for (int R = 0; R < nsub; ++R) {
            if (kept[R] == 0) continue;
            for (int m = 0; m < M.nMat; ++m) {
                bool ok = true;
                for (int v = 0; v < nVar; ++v)
                    if (S.qn[(size_t)L * nVar + v] - S.qn[(size_t)R * nVar + v] !=
                        M.cons_diff[(size_t)m + (size_t)v * M.nMat]) { ok = false; break; }
                if (!ok) continue;
                pairs.push_back({L, R, m, toff});
                toff += (long long)S.dim[L] * kept[R];
            }
        }
    }
    if (!d_dense) {
        // the block table of the new matrix: one block per allowed pair
        sp_out->nsub = nsub;
        sp_out->nMat = M.nMat;
        sp_out->kst = kst;
        sp_out->kept = kept;
        sp_out->off.assign((size_t)nsub * nsub * M.nMat, -1);
        long long tot = 0;
        for (const auto& pr : pairs) {
            sp_out->off[((size_t)pr.L * nsub + pr.R) * M.nMat + pr.m] = tot;
            tot += (long long)kept[pr.L] * kept[pr.R];
        }
        sp_out->total = tot;
        NRG_TRY(sp_buf->ensure(sizeof(double) * (size_t)std::max(tot, 1LL)));
        sp_out->data = sp_buf->as<double>();
    }
    if (pairs.empty()) return NRG_OK;
    DevBuf& T = ctx->scratch.b[6];
    NRG_TRY(T.ensure(sizeof(double) * (size_t)toff));
    NRG_TRY(run_fill(ctx, T.as<double>(), toff, 0.0));
    std::vector<GemmProblem> p1, p2;
    const int* dl = S.d_lst.as<int>();
    for (const auto& pr : pairs) {
        const int L = pr.L, R = pr.R, m = pr.m;
        for (int a = 0; a < nOps; ++a) {
            const int cL = S.cnt(L, a), cR = S.cnt(R, a);
            if (cL == 0 || cR == 0) continue;
            // C(i in L, j in R) = cspec(m, a) IMS_old(ref_j, ref_i, m): rows ref_j, columns ref_i
            long long sr = 0, sl = 0;
            bool bad = false;
            const double* a0 = old.at(S.refBase[(size_t)R * nOps + a], S.refBase[(size_t)L * nOps + a], m, cR, cL,
                                      &sr, &sl, &bad);
            if (bad) {
                nrg_set_error_message("basis_input references outside the previous d-dagger matrix");
                return NRG_ERR_INVALID;
            }
            if (!a0) continue;   // a zero block of the previous matrix
            GemmProblem P;
            std::memset(&P, 0, sizeof(P));
            P.M = cL; P.N = kept[R]; P.K = cR;
            P.alpha = M.cspec[(size_t)m + (size_t)a * M.nMat]; P.beta = 0.0;
            P.A = a0; P.a_si = sl; P.a_sk = sr;
            P.B = d_V + S.ce[R]; P.b_ki = dl + S.lstOff[(size_t)R * nOps + a]; P.b_sk = 1; P.b_sj = S.dim[R];
            P.C = T.as<double>() + pr.t_off; P.c_ri = dl + S.lstOff[(size_t)L * nOps + a];
            P.c_si = 1; P.c_sj = S.dim[L];
            p1.push_back(P);
        }
        GemmProblem Q;
        std::memset(&Q, 0, sizeof(Q));
        Q.M = kept[L]; Q.N = kept[R]; Q.K = S.dim[L];
        Q.alpha = 1.0; Q.beta = 0.0;
        Q.A = d_V + S.ce[L]; Q.a_si = S.dim[L]; Q.a_sk = 1;
        Q.B = T.as<double>() + pr.t_off; Q.b_sk = 1; Q.b_sj = S.dim[L];
        if (d_dense) {
            Q.C = d_dense + kst[R] + kst[L] * nbk + (long long)m * nbk * nbk; Q.c_si = nbk; Q.c_sj = 1;
        } else {
            Q.C = sp_buf->as<double>() + sp_out->off[((size_t)L * nsub + R) * M.nMat + m];
            Q.c_si = kept[R]; Q.c_sj = 1;
        }
        p2.push_back(Q);
    }
    NRG_TRY(launch_ggemm(ctx, p1, 8));
    return launch_ggemm(ctx, p2, 10);
}

// ------------------------------------------------------------------------------------
// backward reduced density matrix step (reducedDensityMatrixDGEMM.F90:115-321)
// ------------------------------------------------------------------------------------
int rdm_step_device(nrg_context* ctx, const IterView& P, const IterView& C, double* d_rdm,
                    double* d_trace_out) {
    const Model& M = ctx->model;
    const Sectors& SP = *P.S;
    const Sectors& SC = *C.S;
    const int nVar = SP.nVar, nOps = SP.nOps;
    struct Blk { int s; int n; long long off; };
    std::vector<Blk> blocks;
    std::vector<GemmProblem> p1;
    std::vector<std::vector<GemmProblem>> p2(nOps);
    std::vector<long long> toffs;
    long long ttot = 0;
    DevBuf& T = ctx->scratch.b[6];
    // first pass: sizes
    struct Link { int S, c, op; long long colOff; };
    std::vector<Link> links;
    std::vector<long long> tS(SP.nsub, -1);
    std::vector<int> q(nVar);
    for (int s = 0; s < SP.nsub; ++s) {
        const int n = P.kept[s];
        if (n == 0) continue;
        long long colOff = 0;
        for (int op = 0; op < nOps; ++op) {
            for (int v = 0; v < nVar; ++v) q[v] = SP.qn[(size_t)s * nVar + v] - M.op(op, v);
            const int c = SC.find(q.data());
            // a child contributes its kept block and, with weights, its discarded columns
            if (c < 0 || (C.kept[c] == 0 && (!C.d_P || SC.dim[c] == C.kept[c]))) continue;
            if (SC.cnt(c, op) != n) {
                nrg_set_error_message("rdm: child sector rows (%d) differ from kept states (%d)",
                                      SC.cnt(c, op), n);
                return NRG_ERR_INVALID;
            }
            links.push_back({s, c, op, colOff});
            colOff += C.d_P ? SC.dim[c] : C.kept[c];
        }
        tS[s] = ttot;
        ttot += (long long)n * colOff;
        blocks.push_back({s, n, P.rdm_off[s]});
    }
    NRG_TRY(T.ensure(sizeof(double) * (size_t)std::max(ttot, 1LL)));
    const int* dl = SC.d_lst.as<int>();
    std::vector<ScaledGather> sg;
    std::vector<GemmProblem> p3;
    for (const auto& lk : links) {
        const int n = P.kept[lk.S], c = lk.c, kc = C.kept[c], dc = SC.dim[c];
        const int* rows = dl + SC.lstOff[(size_t)c * nOps + lk.op];
        if (C.d_P && dc > kc) {
            // discarded columns of the child with their weights: rho_S += (A_D diag(P)) A_D^T
            const long long toff = tS[lk.S] + (lk.colOff + kc) * n;
            sg.push_back({toff, SC.ce[c], SC.lstOff[(size_t)c * nOps + lk.op], SC.start[c] + kc, n, dc - kc, dc, kc});
            GemmProblem D;
            std::memset(&D, 0, sizeof(D));
            D.M = n; D.N = n; D.K = dc - kc; D.alpha = 1.0; D.beta = 1.0;
            D.A = T.as<double>() + toff; D.a_si = 1; D.a_sk = n;
            D.B = C.d_V + SC.ce[c] + (long long)kc * dc; D.b_sk = dc; D.b_ji = rows; D.b_sj = 1;
            D.C = d_rdm + P.rdm_off[lk.S]; D.c_si = n; D.c_sj = 1;
            p3.push_back(D);
        }
        if (kc == 0) continue;
        // T_op = A_op rho_c, A_op(i, k) = V_c(rows[i], k); rho_c row-major
        GemmProblem A;
        std::memset(&A, 0, sizeof(A));
        A.M = n; A.N = kc; A.K = kc; A.alpha = 1.0; A.beta = 0.0;
        A.A = C.d_V + SC.ce[c]; A.a_ri = rows; A.a_si = 1; A.a_sk = dc;
        A.B = d_rdm + C.rdm_off[c]; A.b_sk = kc; A.b_sj = 1;
        A.C = T.as<double>() + tS[lk.S] + lk.colOff * n; A.c_si = 1; A.c_sj = n;
        p1.push_back(A);
        // rho_S += T_op A_op^T (row-major store)
        GemmProblem B;
        std::memset(&B, 0, sizeof(B));
        B.M = n; B.N = n; B.K = kc; B.alpha = 1.0; B.beta = 1.0;
        B.A = T.as<double>() + tS[lk.S] + lk.colOff * n; B.a_si = 1; B.a_sk = n;
        B.B = C.d_V + SC.ce[c]; B.b_sk = dc; B.b_ji = rows; B.b_sj = 1;
        B.C = d_rdm + P.rdm_off[lk.S]; B.c_si = n; B.c_sj = 1;
        p2[lk.op].push_back(B);
    }
    for (const auto& b : blocks) NRG_TRY(run_fill(ctx, d_rdm + b.off, (long long)b.n * b.n, 0.0));
    NRG_TRY(launch_ggemm(ctx, p1, 8));
    for (int op = 0; op < nOps; ++op) NRG_TRY(launch_ggemm(ctx, p2[op], 10));
    if (!sg.empty()) {
        NRG_TRY(run_scaled_gather(ctx, sg, T.as<double>(), C.d_V, dl, C.d_P));
        // the products of one parent block are added one launch after another
        std::vector<std::vector<GemmProblem>> byop(nOps);
        std::vector<int> cnt(SP.nsub, 0);
        for (const auto& D : p3) {
            int s = 0;
            for (const auto& b : blocks)
                if (d_rdm + b.off == D.C) { s = b.s; break; }
            byop[cnt[s]++].push_back(D);
        }
        for (int op = 0; op < nOps; ++op) NRG_TRY(launch_ggemm(ctx, byop[op], 14));
    }
    if (d_trace_out && !blocks.empty()) {
        std::vector<long long> offs;
        std::vector<int> dims;
        for (const auto& b : blocks) { offs.push_back(b.off); dims.push_back(b.n); }
        DevBuf& bo = ctx->scratch.b[12];
        DevBuf& bd = ctx->scratch.b[13];
        NRG_TRY(bo.ensure(sizeof(long long) * offs.size()));
        NRG_TRY(bd.ensure(sizeof(int) * dims.size()));
        NRG_TRY(h2d_async(ctx, bo.p, offs.data(), sizeof(long long) * offs.size()));
        NRG_TRY(h2d_async(ctx, bd.p, dims.data(), sizeof(int) * dims.size()));
        NRG_TRY(run_trace(ctx, d_rdm, bo.as<long long>(), bd.as<int>(), (int)blocks.size(), d_trace_out));
    }
    return NRG_OK;
}

// ------------------------------------------------------------------------------------
// spectrum: spikeCFS (calculateSpectrumDGEMM.F90:217-646) and spikeZeroTemperature (:1-215)
// ------------------------------------------------------------------------------------
namespace {

struct SpecJob {
    int k, l;          // k sector (kept columns / all columns at T=0), l sector
    int kk, c0, nl;    // columns of k used, first l column, number of l columns
    int m, part;       // part 0: <k|d^dag|l>, part 1: <l|d^dag|k>
    double sgn, cE, invpf;
    int toPos;
    long long rdm_off; // -1: T=0 weights
    long long t_off, s_off, y_off;
    int kc0 = 0;       // first k column (discarded-discarded jobs)
    int fdm = 0;       // full-density-matrix weights
};

int run_spec_jobs(nrg_context* ctx, const IterView& it, std::vector<SpecJob>& jobs, const OpView& old,
                  double sc, int nbin, double* d_binPos, double* d_binNeg, double* d_tot) {
    const Model& M = ctx->model;
    const Sectors& S = *it.S;
    const int nOps = S.nOps;
    long long ttot = 0, stot = 0;
    for (auto& j : jobs) {
        j.t_off = ttot;
        ttot += (long long)S.dim[j.k] * j.nl;
        j.s_off = stot;
        stot += (long long)j.kk * j.nl;
        if (j.rdm_off >= 0) { j.y_off = stot; stot += (long long)j.kk * j.nl; } else j.y_off = -1;
    }
    if (jobs.empty()) return NRG_OK;
    DevBuf& T = ctx->scratch.b[6];
    DevBuf& W = ctx->scratch.b[7];
    NRG_TRY(T.ensure(sizeof(double) * (size_t)std::max(ttot, 1LL)));
    NRG_TRY(W.ensure(sizeof(double) * (size_t)std::max(stot, 1LL)));
    NRG_TRY(run_fill(ctx, T.as<double>(), ttot, 0.0));
    const int* dl = S.d_lst.as<int>();
    std::vector<GemmProblem> p1, p2, p3;
    for (const auto& j : jobs) {
        const int k = j.k, l = j.l, m = j.m;
        for (int a = 0; a < nOps; ++a) {
            const int ck = S.cnt(k, a), cl = S.cnt(l, a);
            if (ck == 0 || cl == 0) continue;
            const long long rk = S.refBase[(size_t)k * nOps + a], rl = S.refBase[(size_t)l * nOps + a];
            long long sr = 0, sc2 = 0;
            bool bad = false;
            // part 0: C(i in k, j in l) = cspec(m, a) IMS(ref_j, ref_i, m), rows ref_j (l);
            // part 1: C'(j in k, i in l)^T = IMS(ref_j(k), ref_i(l), m), rows ref_j (k)
            const double* a0 = j.part == 0 ? old.at(rl, rk, m, cl, ck, &sr, &sc2, &bad)
                                           : old.at(rk, rl, m, ck, cl, &sr, &sc2, &bad);
            if (bad) {
                nrg_set_error_message("basis_input references outside the previous d-dagger matrix");
                return NRG_ERR_INVALID;
            }
            if (!a0) continue;   // a zero block of the previous matrix
            GemmProblem P;
            std::memset(&P, 0, sizeof(P));
            P.M = ck; P.N = j.nl; P.K = cl;
            P.alpha = M.cspec[(size_t)m + (size_t)a * M.nMat]; P.beta = 0.0;
            P.A = a0;
            if (j.part == 0) { P.a_si = sc2; P.a_sk = sr; } else { P.a_si = sr; P.a_sk = sc2; }
            P.B = it.d_V + S.ce[l] + (long long)j.c0 * S.dim[l];
            P.b_ki = dl + S.lstOff[(size_t)l * nOps + a]; P.b_sk = 1; P.b_sj = S.dim[l];
            P.C = T.as<double>() + j.t_off; P.c_ri = dl + S.lstOff[(size_t)k * nOps + a];
            P.c_si = 1; P.c_sj = S.dim[k];
            p1.push_back(P);
        }
        GemmProblem Q;
        std::memset(&Q, 0, sizeof(Q));
        Q.M = j.kk; Q.N = j.nl; Q.K = S.dim[k]; Q.alpha = 1.0; Q.beta = 0.0;
        Q.A = it.d_V + S.ce[k] + (long long)j.kc0 * S.dim[k]; Q.a_si = S.dim[k]; Q.a_sk = 1;
        Q.B = T.as<double>() + j.t_off; Q.b_sk = 1; Q.b_sj = S.dim[k];
        Q.C = W.as<double>() + j.s_off; Q.c_si = 1; Q.c_sj = j.kk;
        p2.push_back(Q);
        if (j.rdm_off >= 0) {
            // Y(k1, l) = sum_k2 rho(k2, k1) S(k2, l); rho row-major -> X(k1,k2) = rdm[k1 + kk*k2]
            GemmProblem Y;
            std::memset(&Y, 0, sizeof(Y));
            Y.M = j.kk; Y.N = j.nl; Y.K = j.kk; Y.alpha = 1.0; Y.beta = 0.0;
            Y.A = it.d_rdm + j.rdm_off; Y.a_si = 1; Y.a_sk = j.kk;
            Y.B = W.as<double>() + j.s_off; Y.b_sk = 1; Y.b_sj = j.kk;
            Y.C = W.as<double>() + j.y_off; Y.c_si = 1; Y.c_sj = j.kk;
            p3.push_back(Y);
        }
    }
    NRG_TRY(launch_ggemm(ctx, p1, 8));
    NRG_TRY(launch_ggemm(ctx, p2, 10));
    NRG_TRY(launch_ggemm(ctx, p3, 14));
    std::vector<SpikeProb> sp;
    for (const auto& j : jobs) {
        SpikeProb s;
        s.s_off = j.s_off; s.y_off = j.y_off;
        s.ek_off = S.start[j.k] + j.kc0;
        s.el_off = S.start[j.l] + j.c0;
        s.kk = j.kk; s.nl = j.nl; s.m = j.m; s.toPos = j.toPos; s.lstride = 1;
        s.sgn = j.sgn; s.cE = j.cE; s.scale = sc; s.invpf = j.invpf;
        s.fdm = j.fdm; s.k_is_y = j.part == 0 ? 1 : 0;
        sp.push_back(s);
    }
    return run_spikes(ctx, sp, W.as<double>(), it.d_Esec, nbin, M.nMat, d_binPos, d_binNeg, d_tot, it.d_P);
}

}  // namespace

namespace {
// spikeCFS jobs (calculateSpectrumDGEMM.F90:364-536): every discarded block l with the kept
// sector k = l + positive / negative operation of matrix type m
std::vector<SpecJob> cfs_jobs(const Model& M, const IterView& it) {
    const Sectors& S = *it.S;
    const int nVar = S.nVar;
    std::vector<SpecJob> jobs;
    std::vector<int> q(nVar);
    for (int l = 0; l < S.nsub; ++l) {
        const int nl = S.dim[l] - it.kept[l];
        if (nl <= 0) continue;
        for (int part = 0; part < 2; ++part) {
            const std::vector<int>& ops = part == 0 ? M.pos_op : M.neg_op;
            for (int m = 0; m < M.nMat; ++m) {
                for (int v = 0; v < nVar; ++v) q[v] = S.qn[(size_t)l * nVar + v] + ops[(size_t)m + (size_t)v * M.nMat];
                const int k = S.find(q.data());
                if (k < 0 || it.kept[k] == 0) continue;   // findFullSubspace (:396, :475)
                SpecJob j;
                j.k = k; j.l = l; j.kk = it.kept[k]; j.c0 = it.kept[l]; j.nl = nl; j.m = m;
                j.part = part;
                j.sgn = part == 0 ? 1.0 : -1.0;  // (E_k1 - E_l) (:442) | (E_l - E_k1) (:519)
                j.cE = 1.0;
                j.invpf = 0.0;
                j.toPos = part;                  // negative bins (:458) | positive bins (:532)
                j.rdm_off = it.rdm_off[k];
                jobs.push_back(j);
            }
        }
    }
    return jobs;
}

// spikeZeroTemperature jobs (calculateSpectrumDGEMM.F90:56-211): per ground-state sector,
// the excited sector of each matrix type and sign
std::vector<SpecJob> t0_jobs(const Model& M, const IterView& it, const std::vector<int>& gs_sectors) {
    const Sectors& S = *it.S;
    const int nVar = S.nVar;
    const double pf = (double)gs_sectors.size();
    std::vector<SpecJob> jobs;
    std::vector<int> q(nVar);
    for (int g : gs_sectors) {
        if (g < 0 || g >= S.nsub) continue;
        for (int part = 0; part < 2; ++part) {
            const std::vector<int>& ops = part == 0 ? M.pos_op : M.neg_op;
            for (int m = 0; m < M.nMat; ++m) {
                for (int v = 0; v < nVar; ++v) q[v] = S.qn[(size_t)g * nVar + v] + ops[(size_t)m + (size_t)v * M.nMat];
                const int e = S.find(q.data());
                if (e < 0) continue;
                SpecJob j;
                j.k = e; j.l = g; j.kk = S.dim[e]; j.c0 = 0; j.nl = 1; j.m = m;
                j.part = part;
                j.sgn = part == 0 ? 1.0 : -1.0;   // +E_ex (:154) | -E_ex (:200)
                j.cE = 0.0;
                j.invpf = 1.0 / pf;
                j.toPos = part == 0 ? 1 : 0;
                j.rdm_off = -1;
                jobs.push_back(j);
            }
        }
    }
    return jobs;
}
}  // namespace

std::vector<HostSeg> spike_ims_segs(const Model& M, const IterView& it, const std::vector<int>* gs_sectors,
                                    int nb_old) {
    const Sectors& S = *it.S;
    const int nOps = S.nOps;
    const long long nbo = nb_old;
    const std::vector<SpecJob> jobs = gs_sectors ? t0_jobs(M, it, *gs_sectors) : cfs_jobs(M, it);
    std::vector<HostSeg> segs;
    std::unordered_set<long long> seen;   // segments already listed
    for (const auto& j : jobs)
        for (int a = 0; a < nOps; ++a) {
            const int ck = S.cnt(j.k, a), cl = S.cnt(j.l, a);
            if (ck == 0 || cl == 0) continue;
            const long long rk = S.refBase[(size_t)j.k * nOps + a], rl = S.refBase[(size_t)j.l * nOps + a];
            if (rk < 0 || rl < 0 || rk + ck > nbo || rl + cl > nbo) continue;   // rejected by run_spec_jobs
            // part 0 reads IMS(rows of l, columns of k, m), part 1 IMS(rows of k, columns of l, m)
            const long long r0 = j.part == 0 ? rl : rk, c0 = j.part == 0 ? rk : rl;
            const int nr = j.part == 0 ? cl : ck, nc = j.part == 0 ? ck : cl;
            const long long key = ((long long)j.m * nbo + c0) * nbo + r0;
            if (!seen.insert(key).second) continue;
            segs.push_back({r0 + c0 * nbo + (long long)j.m * nbo * nbo, nr, nc});
        }
    return segs;
}

int spike_cfs_device(nrg_context* ctx, int iteration, const IterView& it, const OpView& old,
                     const double* d_rdm, double* d_binPos, double* d_binNeg, double* d_tot) {
    const Model& M = ctx->model;
    (void)d_rdm;
    std::vector<SpecJob> jobs = cfs_jobs(M, it);
    return run_spec_jobs(ctx, it, jobs, old, M.scale(iteration), M.numberOfBin(), d_binPos, d_binNeg, d_tot);
}

int spike_fdm_device(nrg_context* ctx, int iteration, const IterView& it, const OpView& old,
                     bool last, double* d_binPos, double* d_binNeg, double* d_tot) {
    const Model& M = ctx->model;
    const Sectors& S = *it.S;
    const int nVar = S.nVar;
    std::vector<SpecJob> jobs;
    // kept-discarded pairs: the CFS products, the discarded state's weight added to the
    // kept-space density term; every job once per sign of the bins
    if (!last)
        for (SpecJob j : cfs_jobs(M, it))
            for (int pos = 0; pos < 2; ++pos) {
                j.fdm = 1;
                j.toPos = pos;
                jobs.push_back(j);
            }
    // discarded-discarded pairs: y = x + positive operation of m, <y|d^dag|x> over the
    // discarded columns of both (every column at the last shell)
    auto first_d = [&](int s) { return last ? 0 : it.kept[s]; };
    std::vector<int> q(nVar);
    for (int x = 0; x < S.nsub; ++x) {
        const int dx = S.dim[x] - first_d(x);
        if (dx <= 0) continue;
        for (int m = 0; m < M.nMat; ++m) {
            for (int v = 0; v < nVar; ++v) q[v] = S.qn[(size_t)x * nVar + v] + M.pos_op[(size_t)m + (size_t)v * M.nMat];
            const int y = S.find(q.data());
            if (y < 0) continue;
            const int dy = S.dim[y] - first_d(y);
            if (dy <= 0) continue;
            SpecJob j;
            j.k = y; j.kc0 = first_d(y); j.kk = dy;
            j.l = x; j.c0 = first_d(x); j.nl = dx;
            j.m = m; j.part = 0; j.sgn = 1.0; j.cE = 1.0; j.invpf = 0.0; j.rdm_off = -1; j.fdm = 1;
            for (int pos = 0; pos < 2; ++pos) {
                j.toPos = pos;
                jobs.push_back(j);
            }
        }
    }
    return run_spec_jobs(ctx, it, jobs, old, M.scale(iteration), M.numberOfBin(), d_binPos, d_binNeg, d_tot);
}

int spike_t0_device(nrg_context* ctx, int iteration, const IterView& it,
                    const std::vector<int>& gs_sectors, const OpView& old,
                    double* d_binPos, double* d_binNeg) {
    const Model& M = ctx->model;
    std::vector<SpecJob> jobs = t0_jobs(M, it, gs_sectors);
    DevBuf& tot = ctx->scratch.b[22];
    NRG_TRY(tot.ensure(sizeof(double) * 2 * std::max(M.nMat, 1)));
    return run_spec_jobs(ctx, it, jobs, old, M.scale(iteration), M.numberOfBin(), d_binPos, d_binNeg,
                         tot.as<double>());
}

}  // namespace nrg
