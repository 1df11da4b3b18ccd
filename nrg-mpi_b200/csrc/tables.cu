// Per-state bookkeeping of the device-resident run on the device: the truncation of
// postprocess.F90:69-140 and the next iteration's basis records and row lists of
// prepareBasis.F90:31-114, computed from the eigenvalues where they already are.  The host
// keeps only sector-level tables (quantum numbers, dimensions, kept counts: a few integers
// per sector and operation), which it needs anyway to size the next launches.
//
// Truncation.  postprocess sorts the eigenvalues (sortWithIndex, :75), takes
// Ecut = E(N_keep) + 1e-6, extends the kept count over E <= Ecut (:91-106) and, while the
// count exceeds limit = int(1.2 N_keep), lowers Ecut by 0.001 and peels the states above it
// from the top (:108-124).  On the sorted list the extension gives count(E <= Ecut), and
// every peel gives count(E <= Ecut) for the lowered Ecut; the loop runs while that count
// exceeds limit, i.e. while the (limit+1)-th smallest energy is <= Ecut.  So the kept set
// is {E <= Ecut_final}: two order statistics (the N_keep-th and the (limit+1)-th smallest
// energy, by radix selection) and the same scalar sequence of Ecut values, with no sort.
// The kept states of a sector are its lowest (the eigensolver returns each sector's
// eigenvalues in ascending order, which the kernel checks), so the kept set is one count
// per sector, and sortByIndex (:140) puts them first in sector order.
//
// Basis records.  After the first iteration every record of basis_output is
// (qn of its sector, column in the sector): the kept states of sector s are columns
// 1..k_s.  prepareBasis then forms, for old state i of sector s and operation a, the
// record (qn_s - op_a, reference i, variation = column, operation a) and sorts by
// (qn, reference) (sortBasisArray, module.F90:531-602).  When the operations change the
// quantum numbers in pairwise different ways no two records share (qn, reference), the
// exchange sort's result is the sorted order, and each new sector is the concatenation of
// whole runs (old sector s, operation a) in increasing s: the sector table follows from
// the (s, a) pairs alone, and the records and (sector, operation) row lists are written
// per row by one kernel.  Models whose operations share quantum numbers (the two-orbital
// model) keep the host replay of the exchange sort.
#include "internal.hpp"

#include <algorithm>
#include <numeric>

namespace nrg {
namespace {

// energies as unsigned keys with the numerical order (-0.0 counted as +0.0), the order
// the host's stable sort uses
__device__ __forceinline__ unsigned long long energy_key(double x) {
    if (x == 0.0) x = 0.0;
    const unsigned long long b = (unsigned long long)__double_as_longlong(x);
    return (b >> 63) ? ~b : (b | (1ULL << 63));
}
__device__ __forceinline__ double key_energy(unsigned long long k) {
    const unsigned long long b = (k >> 63) ? (k & ~(1ULL << 63)) : ~k;
    return __longlong_as_double((long long)b);
}

constexpr int kTruncThreads = 1024;

struct TruncShared {
    unsigned hist[256];
    unsigned long long prefix;
    int rank;
    double ecut;
    int status;
};

// The (k+1)-th smallest of E[0, n), 0 <= k < n: most-significant-digit radix selection on
// the energy keys, 8 bits per pass; lanes of a warp that fall in the same bucket add once.
__device__ double select_energy(const double* __restrict__ E, int n, int k, TruncShared& sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();   // every thread has read the previous selection's result
    if (threadIdx.x == 0) {
        sh.prefix = 0;
        sh.rank = k;
    }
    unsigned long long mask = 0;
    for (int shift = 56; shift >= 0; shift -= 8) {
        for (int b = threadIdx.x; b < 256; b += blockDim.x) sh.hist[b] = 0;
        __syncthreads();
        const unsigned long long pre = sh.prefix;
        for (int base = warp * 32; base < n; base += blockDim.x) {
            const int i = base + lane;
            unsigned long long key = 0;
            const bool in = i < n && (((key = energy_key(E[i])) & mask) == pre);
            const unsigned act = __ballot_sync(0xffffffffu, in);
            if (in) {
                const unsigned dig = (unsigned)(key >> shift) & 255u;
                const unsigned peers = __match_any_sync(act, dig);
                if (lane == __ffs(peers) - 1) atomicAdd(&sh.hist[dig], (unsigned)__popc(peers));
            }
        }
        __syncthreads();
        if (warp == 0) {   // the bucket holding rank k: lane l owns buckets 8l .. 8l+7
            unsigned c[8], tot = 0;
            for (int u = 0; u < 8; ++u) { c[u] = sh.hist[8 * lane + u]; tot += c[u]; }
            unsigned incl = tot;
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += v;
            }
            const unsigned rk = (unsigned)sh.rank;
            const unsigned hit = __ballot_sync(0xffffffffu, incl > rk);
            const int owner = __ffs(hit) - 1;   // hit != 0: the buckets hold every candidate
            if (lane == owner) {
                unsigned cum = incl - tot;
                int dig = 8 * lane + 7;
                for (int u = 0; u < 8; ++u) {
                    if (cum + c[u] > rk) { dig = 8 * lane + u; break; }
                    cum += c[u];
                }
                sh.rank = (int)(rk - cum);
                sh.prefix = pre | ((unsigned long long)dig << shift);
            }
        }
        mask |= 255ULL << shift;
        __syncthreads();
    }
    return key_energy(sh.prefix);
}

// One block.  out[0]: kept states; out[1]: status (bit 1: a sector's kept states are not
// its lowest columns; bit 2: the cut-back loop passed its bound); out[2 + s]: kept states of
// sector s.  koff[s]: kept states before sector s (s = 0 .. nsub).  secTab: start (0-based
// row) and dimension of every sector, in sector order.
__global__ void __launch_bounds__(kTruncThreads) k_truncate(const double* __restrict__ E,
                                                            const int* __restrict__ secTab, TruncParams P,
                                                            int* __restrict__ out, int* __restrict__ koff,
                                                            double* __restrict__ ecut_out) {
    __shared__ TruncShared sh;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    const int* start = secTab;
    const int* dim = secTab + P.nsub;
    if (threadIdx.x == 0) sh.status = 0;
    __syncthreads();
    double ecut = INFINITY;
    if (P.truncate) {
        const double en = select_energy(E, P.nb, P.ntrunc - 1, sh);   // E(N_keep) of the sorted list
        double e = en + P.thr;
        if (P.nb > P.limit) {
            const double el = select_energy(E, P.nb, P.limit, sh);    // the (limit+1)-th smallest
            if (threadIdx.x == 0) {
                long long steps = 0;
                while (el <= e) {
                    e = e - P.step;
                    if (++steps > P.max_steps) { sh.status |= 2; break; }
                }
                sh.ecut = e;
            }
            __syncthreads();
            e = sh.ecut;
        }
        ecut = e;
    }
    // kept states per sector: E <= ecut, the lowest columns of the sector
    for (int s = warp; s < P.nsub; s += nwarp) {
        const int r0 = start[s], d = dim[s];
        int cnt = 0, last_kept = -1, first_out = d;
        for (int t = lane; t < d; t += 32) {
            const bool k = !P.truncate || E[r0 + t] <= ecut;
            if (k) { ++cnt; last_kept = t; }
            else first_out = min(first_out, t);
        }
        for (int o = 16; o > 0; o >>= 1) {
            cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
            last_kept = max(last_kept, __shfl_xor_sync(0xffffffffu, last_kept, o));
            first_out = min(first_out, __shfl_xor_sync(0xffffffffu, first_out, o));
        }
        if (lane == 0) {
            out[2 + s] = cnt;
            if (last_kept > first_out) atomicOr(&sh.status, 1);
        }
    }
    __syncthreads();
    if (warp == 0) {   // exclusive prefix over the sectors
        int carry = 0;
        for (int base = 0; base < P.nsub; base += 32) {
            const int s = base + lane;
            const int v = s < P.nsub ? out[2 + s] : 0;
            int incl = v;
            for (int o = 1; o < 32; o <<= 1) {
                const int u = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += u;
            }
            if (s < P.nsub) koff[s] = carry + incl - v;
            carry += __shfl_sync(0xffffffffu, incl, 31);
        }
        if (lane == 0) {
            koff[P.nsub] = carry;
            out[0] = carry;
            out[1] = sh.status;
            ecut_out[0] = ecut;
        }
    }
}

// Eold of the next iteration: the kept (lowest) energies of every sector, in sector order
__global__ void k_gather_kept(const double* __restrict__ E, const int* __restrict__ secTab, int nsub,
                              const int* __restrict__ kept, const int* __restrict__ koff,
                              double* __restrict__ Enext) {
    const int s = blockIdx.x;
    if (s >= nsub) return;
    const int r0 = secTab[s], k = kept[s], o = koff[s];
    for (int t = threadIdx.x; t < k; t += blockDim.x) Enext[o + t] = E[r0 + t];
}

// basis_input records (reference, variation, operation; the quantum-number words stay 0,
// nothing reads them on the device) and the (sector, operation) row lists, one thread per
// row; the runs cover the rows in order
__global__ void k_rows(const RowRun* __restrict__ runs, int nruns, int nb, int rec, int nVar,
                       int* __restrict__ bi, int* __restrict__ lst) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nb;
         i += (long long)gridDim.x * blockDim.x) {
        int lo = 0, hi = nruns - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (runs[mid].row0 <= i) lo = mid; else hi = mid - 1;
        }
        const RowRun r = runs[lo];
        const int t = (int)(i - r.row0);
        int* b = bi + (size_t)i * rec;
        for (int v = 0; v < nVar; ++v) b[v] = 0;
        b[nVar] = r.ref0 + t + 1;
        b[nVar + 1] = t + 1;
        b[nVar + 2] = r.op + 1;
        lst[r.lst0 + t] = (int)(i - r.sec_start);
    }
}

}  // namespace

bool ops_change_qn_distinctly(const Model& M) {
    for (int a = 0; a < M.nOps; ++a)
        for (int b = a + 1; b < M.nOps; ++b) {
            bool eq = true;
            for (int v = 0; v < M.nVar && eq; ++v) eq = M.op(a, v) == M.op(b, v);
            if (eq) return false;
        }
    return true;
}

int Sectors::plan(const Model& M, const Sectors& prev, const std::vector<int>& kept_prev,
                  std::vector<RowRun>* runs) {
    nVar = M.nVar;
    nOps = M.nOps;
    const int np = prev.nsub;
    if ((int)kept_prev.size() != np || prev.nVar != nVar) {
        nrg_set_error_message("sector plan: inconsistent previous table");
        return NRG_ERR_INVALID;
    }
    std::vector<long long> koff(np + 1, 0);
    for (int s = 0; s < np; ++s) koff[s + 1] = koff[s] + kept_prev[s];
    if (koff[np] * nOps > 0x7fffffffLL) {
        nrg_set_error_message("sector plan: %lld basis states exceed 32-bit indices", koff[np] * nOps);
        return NRG_ERR_TOO_LARGE;
    }
    // the (old sector, operation) pairs in generation order, then stably by quantum numbers:
    // within one set of quantum numbers the old sectors keep their order, i.e. the order of
    // their references
    std::vector<int> key;
    std::vector<int> pairS, pairA;
    for (int s = 0; s < np; ++s) {
        if (kept_prev[s] <= 0) continue;
        for (int a = 0; a < nOps; ++a) {
            for (int v = 0; v < nVar; ++v) key.push_back(prev.qn[(size_t)s * nVar + v] - M.op(a, v));
            pairS.push_back(s);
            pairA.push_back(a);
        }
    }
    const int npair = (int)pairS.size();
    std::vector<int> ord(npair);
    std::iota(ord.begin(), ord.end(), 0);
    std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) {
        return std::lexicographical_compare(&key[(size_t)x * nVar], &key[(size_t)x * nVar] + nVar,
                                            &key[(size_t)y * nVar], &key[(size_t)y * nVar] + nVar);
    });
    qn.clear(); dim.clear(); start.clear(); ce.clear();
    runs->clear();
    int row = 0;
    for (int x = 0; x < npair; ++x) {
        const int p = ord[x];
        const int* q = &key[(size_t)p * nVar];
        const bool fresh = x == 0 || !std::equal(q, q + nVar, &key[(size_t)ord[x - 1] * nVar]);
        if (fresh) {
            qn.insert(qn.end(), q, q + nVar);
            dim.push_back(0);
            start.push_back(row);
        } else if (pairS[ord[x - 1]] == pairS[p]) {   // two operations with the same change
            nrg_set_error_message("sector plan: operations %d and %d change the quantum numbers alike",
                                  pairA[ord[x - 1]] + 1, pairA[p] + 1);
            return NRG_ERR_UNSUPPORTED;
        }
        const int sec = (int)dim.size() - 1;
        RowRun r;
        r.row0 = row;
        r.len = kept_prev[pairS[p]];
        r.ref0 = (int)koff[pairS[p]];
        r.op = pairA[p];
        r.sec = sec;
        r.sec_start = start[sec];
        r.lst0 = 0;
        runs->push_back(r);
        dim[sec] += r.len;
        row += r.len;
    }
    nsub = (int)dim.size();
    nb = row;
    long long acc = 0;
    ce.resize(nsub);
    for (int s = 0; s < nsub; ++s) {
        ce[s] = acc;
        acc += (long long)dim[s] * dim[s];
    }
    sizeV = acc;
    // row lists per (sector, operation): one run each (two runs of one operation in one
    // sector would come from two old sectors with the same quantum numbers)
    lstOff.assign((size_t)nsub * nOps + 1, 0);
    refBase.assign((size_t)nsub * nOps, -1);
    for (const RowRun& r : *runs) {
        const size_t k = (size_t)r.sec * nOps + r.op;
        if (refBase[k] >= 0) {
            nrg_set_error_message("sector plan: two previous sectors share quantum numbers");
            return NRG_ERR_INVALID;
        }
        refBase[k] = r.ref0;
        lstOff[k + 1] = r.len;
    }
    for (size_t x = 1; x < lstOff.size(); ++x) lstOff[x] += lstOff[x - 1];
    for (RowRun& r : *runs) r.lst0 = lstOff[(size_t)r.sec * nOps + r.op];
    lst.clear();
    rowOp.clear(); rowRef.clear(); rowVar.clear();
    index_qn();
    return NRG_OK;
}

int rows_device(nrg_context* ctx, Sectors& S, const std::vector<RowRun>& runs) {
    const int rs = S.nVar + 3;
    DevBuf& bRuns = ctx->scratch.b[45];
    NRG_TRY(bRuns.ensure(sizeof(RowRun) * std::max<size_t>(runs.size(), 1)));
    NRG_TRY(S.d_bi.ensure(sizeof(int) * (size_t)S.nb * rs));
    NRG_TRY(S.d_lst.ensure(sizeof(int) * ((size_t)S.nb + 1)));
    NRG_TRY(S.d_lstOff.ensure(sizeof(int) * S.lstOff.size()));
    NRG_TRY(h2d_async(ctx, bRuns.p, runs.data(), sizeof(RowRun) * runs.size()));
    NRG_TRY(h2d_async(ctx, S.d_lstOff.p, S.lstOff.data(), sizeof(int) * S.lstOff.size()));
    if (S.nb == 0 || runs.empty()) return NRG_OK;
    const int threads = 256;
    const long long blocks = std::min<long long>((S.nb + threads - 1) / threads, 148LL * 16);
    k_rows<<<(unsigned)blocks, threads, 0, ctx->stream>>>(bRuns.as<RowRun>(), (int)runs.size(), S.nb, rs, S.nVar,
                                                           S.d_bi.as<int>(), S.d_lst.as<int>());
    ctx->launches++;
    NRG_CUDA_TRY(cudaGetLastError());
    return NRG_OK;
}

int TruncTables::prepare(nrg_context* ctx, const Sectors& S) {
    if (P.truncate && (P.ntrunc < 1 || P.ntrunc > P.nb)) {
        nrg_set_error_message("device truncation: N_keep %d outside 1..%d", P.ntrunc, P.nb);
        return NRG_ERR_INVALID;
    }
    std::vector<int> tab(2 * (size_t)S.nsub);
    for (int s = 0; s < S.nsub; ++s) {
        tab[s] = S.start[s];
        tab[S.nsub + s] = S.dim[s];
    }
    nsub = S.nsub;
    NRG_TRY(ctx->scratch.b[42].ensure(sizeof(int) * std::max<size_t>(tab.size(), 1)));
    const size_t ecut_at = (sizeof(int) * (2 + (size_t)S.nsub) + 7) & ~size_t(7);   // the double after the counts
    NRG_TRY(ctx->scratch.b[43].ensure(ecut_at + sizeof(double)));
    NRG_TRY(ctx->scratch.b[44].ensure(sizeof(int) * ((size_t)S.nsub + 1)));
    NRG_TRY(ctx->h_kept.ensure(sizeof(int) * (2 + (size_t)S.nsub)));
    d_secTab = ctx->scratch.b[42].as<int>();
    d_out = ctx->scratch.b[43].as<int>();
    d_koff = ctx->scratch.b[44].as<int>();
    d_ecut = reinterpret_cast<double*>(ctx->scratch.b[43].as<char>() + ecut_at);
    h_out = ctx->h_kept.as<int>();
    return h2d_async(ctx, d_secTab, tab.data(), sizeof(int) * tab.size());
}

int TruncTables::launch(nrg_context* ctx, const double* d_E) {
    k_truncate<<<1, kTruncThreads, 0, ctx->stream>>>(d_E, d_secTab, P, d_out, d_koff, d_ecut);
    ctx->launches++;
    NRG_CUDA_TRY(cudaGetLastError());
    NRG_CUDA_TRY(cudaMemcpyAsync(h_out, d_out, sizeof(int) * (2 + (size_t)nsub), cudaMemcpyDeviceToHost, ctx->stream));
    ctx->d2h += (long long)sizeof(int) * (2 + nsub);
    return NRG_OK;
}

int TruncTables::result(std::vector<int>* kept, int* nb_kept) const {
    if (h_out[1] != 0) {
        nrg_set_error_message("device truncation: status 0x%x (1: a sector's eigenvalues are not ascending, 2: "
                              "the 0.001 cut-back passed %lld steps)", h_out[1], P.max_steps);
        return (h_out[1] & 2) ? NRG_ERR_NUMERIC : NRG_ERR_INVALID;
    }
    kept->assign(h_out + 2, h_out + 2 + nsub);
    *nb_kept = h_out[0];
    return NRG_OK;
}

int TruncTables::gather(nrg_context* ctx, const double* d_E, double* d_Enext) const {
    if (nsub == 0) return NRG_OK;
    k_gather_kept<<<(unsigned)nsub, 128, 0, ctx->stream>>>(d_E, d_secTab, nsub, d_out + 2, d_koff, d_Enext);
    ctx->launches++;
    NRG_CUDA_TRY(cudaGetLastError());
    return NRG_OK;
}

}  // namespace nrg
