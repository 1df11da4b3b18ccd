// Replay of the reference driver (main.F90:142-252): the forward NRG sweep
// (nrgIteration.F90 -> prepareBasis, diagonalization, postprocess), the backward reduced
// density matrices and the CFS spectrum at T = 0.
//
// Two data flows:
// * device resident (nrg_run_input.host_drop_in = 0): eigenvector blocks, invariant
//   matrices, density matrices and bins stay in device memory, and so does the per-state
//   bookkeeping (the truncation, the next iteration's basis records and row lists, the
//   kept energies: tables.cu); the host keeps the sector-level tables it sizes the
//   launches with (a few integers per sector and operation cross per iteration).  Models
//   whose operations change the quantum numbers alike (ties in sortBasisArray) build the
//   records on the host, with the exchange sort replayed;
// * host drop-in (host_drop_in = 1): every routine goes through its public entry point
//   with host arrays, exactly as the Fortran caller would call the drop-in: module arrays
//   live in host memory and cross to the device and back at every call.
#include "internal.hpp"

#include <chrono>
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

using namespace nrg;

namespace {

// The stable order of the records by (quantum numbers, reference) without comparisons:
// records come in generation order (old state i, operation j), so within one set of
// quantum numbers the references never decrease, and a stable counting sort over the
// distinct quantum numbers (a few hundred) gives the stable sort's order.  Returns false
// (the caller sorts by comparison) when the references do decrease somewhere.
bool bucket_order(const std::vector<int>& rec, int n, int nVar, std::vector<int>* idx) {
    const int rs = nVar + 3;
    std::vector<int> bucket(n);
    std::vector<int> keys;            // distinct quantum numbers, nVar per bucket
    std::vector<int> last_ref;        // reference of the bucket's last record
    std::vector<int> table(64, -1);   // open addressing: bucket per hash slot
    size_t mask = table.size() - 1;
    auto slot_of = [&](const int* q) {
        size_t h = 1469598103934665603ULL;
        for (int v = 0; v < nVar; ++v) h = (h ^ (size_t)(uint32_t)q[v]) * 1099511628211ULL;
        return h;
    };
    for (int r = 0; r < n; ++r) {
        const int* q = &rec[(size_t)r * rs];
        if (2 * keys.size() / nVar >= table.size() / 2) {   // grow and rehash
            table.assign(table.size() * 4, -1);
            mask = table.size() - 1;
            for (int b = 0; b < (int)(keys.size() / nVar); ++b)
                for (size_t x = slot_of(&keys[(size_t)b * nVar]) & mask;; x = (x + 1) & mask)
                    if (table[x] < 0) { table[x] = b; break; }
        }
        int b = -1;
        for (size_t x = slot_of(q) & mask;; x = (x + 1) & mask) {
            if (table[x] < 0) {
                b = (int)(keys.size() / nVar);
                table[x] = b;
                keys.insert(keys.end(), q, q + nVar);
                last_ref.push_back(q[nVar]);
                break;
            }
            if (std::equal(q, q + nVar, &keys[(size_t)table[x] * nVar])) { b = table[x]; break; }
        }
        if (q[nVar] < last_ref[b]) return false;
        last_ref[b] = q[nVar];
        bucket[r] = b;
    }
    const int nb = (int)(keys.size() / nVar);
    std::vector<int> order(nb);
    std::iota(order.begin(), order.end(), 0);
    std::sort(order.begin(), order.end(), [&](int a, int b) {
        return std::lexicographical_compare(&keys[(size_t)a * nVar], &keys[(size_t)a * nVar] + nVar,
                                            &keys[(size_t)b * nVar], &keys[(size_t)b * nVar] + nVar);
    });
    std::vector<int> start(nb + 1, 0), rank(nb);
    for (int k = 0; k < nb; ++k) rank[order[k]] = k;
    for (int r = 0; r < n; ++r) start[rank[bucket[r]] + 1]++;
    for (int k = 0; k < nb; ++k) start[k + 1] += start[k];
    for (int r = 0; r < n; ++r) (*idx)[start[rank[bucket[r]]]++] = r;
    return true;
}

// One pass i of the exchange sequence on ranks R (ids I carried along): the carried key
// is swapped with every strictly smaller key after position i, until it is the pass's
// target (the i-th smallest key), after which no key can be smaller.  ready(e) returns
// once the positions below e hold the previous pass's result; publish(j) announces that
// this pass is done with the positions below j.
template <class Ready, class Publish>
void exchange_pass(int* R, int* I, int n, int i, int t, Ready&& ready, Publish&& publish) {
    ready(i + 1);
    int c = R[i], ci = I[i];
    int j = i + 1;
    while (c > t && j < n) {
        ready(std::min(n, j + 256));
        const int stop = std::min(n, j + 256);
        while (c > t && j < stop) {
            // skip keys not smaller than the carried one, eight at a time
            while (j + 8 <= stop) {
                int m = 0;
                for (int u = 0; u < 8; ++u) m |= R[j + u] < c;
                if (m) break;
                j += 8;
            }
            for (const int end = std::min(stop, j + 8); c > t && j < end; ++j) {
                const int x = R[j];
                if (x < c) {
                    R[j] = c;
                    c = x;
                    const int xi = I[j];
                    I[j] = ci;
                    ci = xi;
                }
            }
        }
        publish(j);
    }
    R[i] = c;
    I[i] = ci;
}

// All passes of the exchange sequence.  Large inputs run consecutive passes on several
// host threads in a wavefront: pass i+1 reads a position only after pass i has moved past
// it (an acquire/release progress word per thread, tagged with the pass number), so every
// swap is the one the serial sequence makes, in the same order per position.
void exchange_replay(int* R, int* I, const int* target, int n) {
    const unsigned hw = std::thread::hardware_concurrency();
    const int T = (int)std::min<unsigned>(8, hw ? hw : 1);
    if (n < 16384 || T < 2) {
        for (int i = 0; i < n; ++i)
            exchange_pass(R, I, n, i, target[i], [](int) {}, [](int) {});
        return;
    }
    // progress word of the pass a thread runs: (pass + 1) << 32 | first position not done
    std::vector<std::atomic<uint64_t>> prog(T);
    for (auto& p : prog) p.store(0, std::memory_order_relaxed);
    auto worker = [&](int k) {
        for (int i = k; i < n; i += T) {
            std::atomic<uint64_t>& mine = prog[k];
            std::atomic<uint64_t>& prev = prog[(k + T - 1) % T];
            int known = i == 0 ? n : 0;      // positions the previous pass is done with
            auto ready = [&](int e) {
                for (int spins = 0; known < e; ++spins) {
                    const uint64_t v = prev.load(std::memory_order_acquire);
                    const long long pass = (long long)(v >> 32) - 1;
                    known = pass > i - 1 ? n : (pass == i - 1 ? (int)(uint32_t)v : 0);
                    if (known < e && spins > 64) std::this_thread::yield();
                }
            };
            auto publish = [&](int j) {
                mine.store(((uint64_t)(i + 1) << 32) | (uint32_t)j, std::memory_order_release);
            };
            publish(i + 1);
            exchange_pass(R, I, n, i, target[i], ready, publish);
            publish(n);
        }
    };
    std::vector<std::thread> pool;
    for (int k = 1; k < T; ++k) pool.emplace_back(worker, k);
    worker(0);
    for (auto& th : pool) th.join();
}

// sortBasisArray (module.F90:531-602): exchange sort of whole records.  When no two
// records share (basis, reference) any correct sort gives its result; otherwise the
// order among equal keys is the exchange sequence's, which is replayed.
void sort_basis(std::vector<int>& rec, int n, int nVar) {
    const int rs = nVar + 3;
    auto greater = [&](const int* a, const int* b) {
        for (int i = 0; i < nVar; ++i) {
            if (a[i] > b[i]) return true;
            if (a[i] < b[i]) return false;
        }
        return a[nVar] > b[nVar];
    };
    std::vector<int> idx(n);
    if (!bucket_order(rec, n, nVar, &idx)) {
        std::iota(idx.begin(), idx.end(), 0);
        std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) {
            return greater(&rec[(size_t)y * rs], &rec[(size_t)x * rs]);
        });
    }
    bool ties = false;
    for (int i = 1; i < n && !ties; ++i) {
        const int* a = &rec[(size_t)idx[i - 1] * rs];
        const int* b = &rec[(size_t)idx[i] * rs];
        ties = !greater(b, a) && !greater(a, b);
    }
    if (!ties) {
        std::vector<int> out((size_t)n * rs);
        for (int i = 0; i < n; ++i) std::memcpy(&out[(size_t)i * rs], &rec[(size_t)idx[i] * rs], sizeof(int) * rs);
        rec.swap(out);
        return;
    }
    // The exchange sequence on integer ranks of the keys (equal keys, equal ranks) with
    // the records' ids carried along.  Pass i carries the smallest key seen so far and
    // swaps it with every strictly smaller key after it; it ends once the carried key is
    // the i-th smallest of all (known from the stable sort above), since no key after it
    // can then be smaller: the same swaps as the full scan, without the tail.
    std::vector<int> rk(n), id(n), target(n);
    for (int k = 0, r = -1; k < n; ++k) {
        if (k == 0 || greater(&rec[(size_t)idx[k] * rs], &rec[(size_t)idx[k - 1] * rs])) ++r;
        rk[idx[k]] = r;
        target[k] = r;
    }
    std::iota(id.begin(), id.end(), 0);
    exchange_replay(rk.data(), id.data(), target.data(), n);
    const int* I = id.data();
    std::vector<int> out((size_t)n * rs);
    for (int i = 0; i < n; ++i) std::memcpy(&out[(size_t)i * rs], &rec[(size_t)I[i] * rs], sizeof(int) * rs);
    rec.swap(out);
}

// prepareBasis (prepareBasis.F90:31-114): product basis, sort, sector table.  Returns the
// count_eigenvector the next sector would get (1 + sum of d^2 over all sectors); a value
// above 2^31 - 1 means the reference's 32-bit field (module.F90:128) cannot hold the
// offsets, and the stored offsets are then capped at 2^31 - 1.
long long prepare_basis_host(const Model& M, const std::vector<int>& bo, int nb_old, std::vector<int>* rec,
                             std::vector<int>* si) {
    const int nVar = M.nVar, rs = nVar + 3, nOps = M.nOps;
    const int nb = nb_old * nOps;
    rec->assign((size_t)nb * rs, 0);
    for (int i = 0; i < nb_old; ++i)
        for (int j = 0; j < nOps; ++j) {
            int* r = &(*rec)[((size_t)i * nOps + j) * rs];
            for (int v = 0; v < nVar; ++v) r[v] = bo[(size_t)i * rs + v] - M.op(j, v);
            r[nVar] = i + 1;
            r[nVar + 1] = bo[(size_t)i * rs + nVar];
            r[nVar + 2] = j + 1;
        }
    sort_basis(*rec, nb, nVar);
    si->clear();
    int s0 = 0;
    long long ce = 1;
    for (int i = 1; i <= nb; ++i) {
        bool brk = (i == nb);
        if (!brk)
            for (int v = 0; v < nVar; ++v)
                if ((*rec)[(size_t)i * rs + v] != (*rec)[(size_t)s0 * rs + v]) { brk = true; break; }
        if (brk) {
            const int d = i - s0;
            for (int v = 0; v < nVar; ++v) si->push_back((*rec)[(size_t)s0 * rs + v]);
            si->push_back(d);
            si->push_back((int)std::min(ce, 0x7fffffffLL));
            si->push_back(s0 + 1);
            ce += (long long)d * d;
            s0 = i;
        }
    }
    return ce;
}

// sortWithIndex + truncation + sortByIndex (postprocess.F90:71-140).  E is indexed by
// row (sector order); returns the kept count and the new order of the rows.
// Stable ascending order of E (std::stable_sort's order under <) by an LSD radix sort on
// the IEEE bit patterns: negative values have every bit flipped, the others the sign bit
// set, so unsigned order is numerical order; -0.0 counts as +0.0 (they compare equal).
// Digits that all keys share are skipped.
void stable_energy_order(const std::vector<double>& E, std::vector<int>* order) {
    const int n = (int)E.size();
    std::vector<uint64_t> key(n);
    for (int i = 0; i < n; ++i) {
        const double x = E[i] == 0.0 ? 0.0 : E[i];
        uint64_t b;
        std::memcpy(&b, &x, sizeof(b));
        key[i] = (b >> 63) ? ~b : (b | (1ULL << 63));
    }
    std::vector<uint32_t> hist(8 * 256, 0);
    for (int i = 0; i < n; ++i)
        for (int d = 0; d < 8; ++d) hist[d * 256 + ((key[i] >> (8 * d)) & 255)]++;
    std::vector<int> a(n), b(n);
    std::iota(a.begin(), a.end(), 0);
    for (int d = 0; d < 8; ++d) {
        uint32_t* h = &hist[d * 256];
        if (h[(key[a[0]] >> (8 * d)) & 255] == (uint32_t)n) continue;   // one bucket: order kept
        uint32_t sum = 0;
        for (int k = 0; k < 256; ++k) {
            const uint32_t c = h[k];
            h[k] = sum;
            sum += c;
        }
        for (int i = 0; i < n; ++i) b[h[(key[a[i]] >> (8 * d)) & 255]++] = a[i];
        a.swap(b);
    }
    order->swap(a);
}

int truncate_host(const Model& M, int it, const std::vector<double>& E, std::vector<int>* order,
                  int* startTrancation, bool* flag_truncation) {
    const int nb = (int)E.size();
    if (nb > 0) stable_energy_order(E, order);
    else order->clear();
    int nbk = nb;
    if (it != M.first && it != M.nIter && nb > M.truncation) {
        if (*startTrancation > it) { *startTrancation = it; *flag_truncation = true; }
        const int limit = (int)(M.truncation * 1.2);
        double Ecut = E[(*order)[M.truncation - 1]];
        int i = M.truncation + 1, cutoff = M.truncation;
        Ecut = Ecut + 0.000001;
        while (i <= nb) {
            if (E[(*order)[i - 1]] <= Ecut) cutoff++; else break;
            ++i;
        }
        while (cutoff > limit) {
            Ecut = Ecut - 0.001;
            for (int q = cutoff; q >= 1; --q) {
                if (E[(*order)[q - 1]] > Ecut) cutoff--; else break;
            }
        }
        nbk = cutoff;
    }
    // sortByIndex on the kept prefix (:140): the kept rows in increasing order
    std::vector<char> kept(nb, 0);
    for (int q = 0; q < nbk; ++q) kept[(*order)[q]] = 1;
    for (int r = 0, q = 0; r < nb; ++r)
        if (kept[r]) (*order)[q++] = r;
    return nbk;
}

void record_flow(nrg_run_output* out, int idx, const std::vector<double>& E, const std::vector<int>& order, int nbk) {
    if (!out || !out->flow || out->flowStride <= 0) return;
    std::vector<double> e(nbk);
    for (int q = 0; q < nbk; ++q) e[q] = E[order[q]];
    const int m = std::min(out->flowStride, nbk);
    std::partial_sort(e.begin(), e.begin() + m, e.end());
    for (int q = 0; q < out->flowStride; ++q)
        out->flow[(size_t)idx * out->flowStride + q] = q < nbk ? e[q] : NAN;
}

// For each sector s of the table si (nsub records of nVar+3 ints): how many of the first
// nbk records of bo carry its quantum numbers, and the index of the first of them (-1
// when none), as the scan of postprocess.F90:303-321 finds them; one pass over the
// records with exact 64-bit keys (up to four 16-bit quantum numbers), the scan itself
// otherwise (or when two sectors share their numbers).
void kept_in_sectors(const std::vector<int>& si, int nsub, const std::vector<int>& bo, int nbk, int nVar,
                     std::vector<int>* count, std::vector<int>* first) {
    const int rs = nVar + 3;
    count->assign(nsub, 0);
    first->assign(nsub, -1);
    auto key = [&](const int* q, uint64_t* k) {
        uint64_t x = 0;
        for (int v = 0; v < nVar; ++v) {
            if (q[v] < -32768 || q[v] > 32767) return false;
            x = (x << 16) | (uint16_t)(int16_t)q[v];
        }
        *k = x;
        return true;
    };
    bool packed = nVar <= 4;
    std::unordered_map<uint64_t, int> sector;
    if (packed) {
        sector.reserve(2 * (size_t)nsub);
        for (int s = 0; s < nsub && packed; ++s) {
            uint64_t k = 0;
            packed = key(&si[(size_t)s * rs], &k) && sector.emplace(k, s).second;
        }
    }
    for (int j = 0; packed && j < nbk; ++j) {
        uint64_t k = 0;
        if (!key(&bo[(size_t)j * rs], &k)) { packed = false; break; }
        const auto it = sector.find(k);
        if (it == sector.end()) continue;
        if ((*first)[it->second] < 0) (*first)[it->second] = j;
        (*count)[it->second]++;
    }
    if (packed) return;
    count->assign(nsub, 0);
    first->assign(nsub, -1);
    for (int s = 0; s < nsub; ++s)
        for (int j = 0; j < nbk; ++j) {
            bool eq = true;
            for (int v = 0; v < nVar; ++v)
                if (si[(size_t)s * rs + v] != bo[(size_t)j * rs + v]) { eq = false; break; }
            if (eq) {
                if ((*first)[s] < 0) (*first)[s] = j;
                (*count)[s]++;
            }
        }
}

// basis_output of the kept states after the first iteration: (qn of the sector, column)
// for columns 1..kept of every sector, in sector order (postprocess.F90:140-160 on the
// record diagonalization.F90:394-407 writes)
std::vector<int> kept_records(const Sectors& S, const std::vector<int>& kept) {
    const int rs = S.nVar + 3;
    std::vector<int> bo;
    for (int s = 0; s < S.nsub; ++s)
        for (int t = 0; t < kept[s]; ++t) {
            const size_t o = bo.size();
            bo.resize(o + rs, 0);
            for (int v = 0; v < S.nVar; ++v) bo[o + v] = S.qn[(size_t)s * S.nVar + v];
            bo[o + S.nVar] = t + 1;
        }
    return bo;
}

bool env_flag(const char* name) {
    const char* v = std::getenv(name);
    return v && std::atoi(v) != 0;
}

// NRG_CHECK_TABLES=1 (a test aid): the tables the device built for one iteration against
// the host's prepareBasis on the same kept states, every sector-level field and every
// downloaded record and row list compared exactly
int check_device_rows(nrg_context* ctx, const Model& M, int it, const Sectors& prev, const std::vector<int>& kept_prev,
                      const Sectors& S) {
    const int rs = M.nVar + 3;
    const std::vector<int> bo = kept_records(prev, kept_prev);
    const int nb_old = (int)(bo.size() / rs);
    std::vector<int> rec, si;
    prepare_basis_host(M, bo, nb_old, &rec, &si);
    Sectors H;
    NRG_TRY(H.build((int)(si.size() / rs), si.data(), nb_old * M.nOps, rec.data(), M.nVar, M.nOps));
    const char* what = nullptr;
    if (H.nsub != S.nsub || H.nb != S.nb) what = "sector or state count";
    else if (H.qn != S.qn || H.dim != S.dim || H.start != S.start || H.ce != S.ce || H.sizeV != S.sizeV)
        what = "sector table";
    else if (H.lstOff != S.lstOff || H.refBase != S.refBase) what = "row-list offsets";
    if (!what) {
        std::vector<int> bi((size_t)S.nb * rs), lst(H.lst.size());
        NRG_CUDA_TRY(cudaMemcpyAsync(bi.data(), S.d_bi.p, sizeof(int) * bi.size(), cudaMemcpyDeviceToHost, ctx->stream));
        if (!lst.empty())
            NRG_CUDA_TRY(cudaMemcpyAsync(lst.data(), S.d_lst.p, sizeof(int) * lst.size(), cudaMemcpyDeviceToHost,
                                         ctx->stream));
        NRG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        if (lst != H.lst) what = "row lists";
        for (int i = 0; i < S.nb && !what; ++i)
            if (bi[(size_t)i * rs + M.nVar] != H.rowRef[i] + 1 || bi[(size_t)i * rs + M.nVar + 1] != H.rowVar[i] ||
                bi[(size_t)i * rs + M.nVar + 2] != H.rowOp[i] + 1)
                what = "basis_input records";
    }
    if (what) {
        nrg_set_error_message("iteration %d: the device-built %s differ from the host's prepareBasis", it, what);
        return NRG_ERR_STATE;
    }
    return NRG_OK;
}

struct IterRec {
    int nb_full = 0, nb_kept = 0;
    double emin = 0.0;   // the minimum the shift subtracted (full-density-matrix energies)
    std::vector<int> kept;
    std::vector<double> Esec;
    std::vector<long long> rdm_off;
};

void write_bins(const Model& M, nrg_run_output* out, int nbin, const double* pos_w, const double* neg_w,
                bool device) {
    const size_t nw = (size_t)nbin * M.nMat;
    for (int m = 0; m < M.nMat; ++m)
        for (int i = 0; i < nbin; ++i) {
            const double e = std::pow(10.0, -15.0 + double(i) / 1000.0);   // main.F90:152-157
            out->binnedSpikePositive[(size_t)m * nbin + i] = e;
            out->binnedSpikeNegative[(size_t)m * nbin + i] = -e;
        }
    if (device) {
        cudaMemcpy(out->binnedSpikePositive + nw, pos_w, sizeof(double) * nw, cudaMemcpyDeviceToHost);
        cudaMemcpy(out->binnedSpikeNegative + nw, neg_w, sizeof(double) * nw, cudaMemcpyDeviceToHost);
    } else {
        std::memcpy(out->binnedSpikePositive + nw, pos_w, sizeof(double) * nw);
        std::memcpy(out->binnedSpikeNegative + nw, neg_w, sizeof(double) * nw);
    }
}

// ------------------------------------------------------------------------------------
// device-resident data flow
// ------------------------------------------------------------------------------------
int run_device(nrg_context* ctx, const nrg_run_input* in, nrg_run_output* out, cudaEvent_t* ev) {
    const Model& M = ctx->model;
    if (in->save_restart || in->load_restart) {
        nrg_set_error_message("restart.dat is written and read by the drop-in replay (host_drop_in = 1)");
        return NRG_ERR_INVALID;
    }
    const int nVar = M.nVar, rs = nVar + 3, first = M.first, nIter = M.nIter;
    const int nIt = nIter - first + 1;
    const bool spectrum = in->spectrum && M.nMat > 0;
    cudaStream_t st = ctx->stream;
    // ---- initial state (read_initial_basis) ----
    int nb_old = in->numberOfBasis;
    std::vector<int> bo(in->basis_output, in->basis_output + (size_t)nb_old * rs);
    DevBuf& bEold0 = ctx->slot(3);
    DevBuf& bIM0 = ctx->slot(1);
    NRG_TRY(bEold0.ensure(sizeof(double) * nb_old));
    NRG_TRY(bIM0.ensure(sizeof(double) * (size_t)nb_old * nb_old * M.nCM));
    NRG_CUDA_TRY(cudaMemcpyAsync(bEold0.p, in->eigenvalue, sizeof(double) * nb_old, cudaMemcpyHostToDevice, st));
    NRG_CUDA_TRY(cudaMemcpyAsync(bIM0.p, in->invariant_matrix, sizeof(double) * (size_t)nb_old * nb_old * M.nCM,
                                 cudaMemcpyHostToDevice, st));
    ctx->h2d += (long long)sizeof(double) * nb_old * (1 + (long long)nb_old * M.nCM);
    const double* dEold = bEold0.as<double>();
    const double* dIMold = bIM0.as<double>();
    // the d-dagger matrices: the initial one dense (initial.dat), those of the iterations
    // block-sparse (only the blocks of allowed sector pairs)
    OpView imsOld;
    std::vector<SparseBlocks> imsTab(nIt);
    if (spectrum) {
        DevBuf& b = ctx->slot(9);
        const size_t n = (size_t)nb_old * nb_old * M.nMat;
        NRG_TRY(b.ensure(sizeof(double) * n));
        NRG_CUDA_TRY(cudaMemcpyAsync(b.p, in->invariant_matrix_spectrum, sizeof(double) * n, cudaMemcpyHostToDevice, st));
        ctx->h2d += (long long)(sizeof(double) * n);
        imsOld.dense = b.as<double>();
        imsOld.nb = nb_old;
    }
    if ((int)ctx->iter_sectors.size() < nIt) ctx->iter_sectors.resize(nIt);
    ctx->slot(22 + 3 * (size_t)nIt);   // size the store once: references below stay valid
    std::vector<IterRec> recs(nIt);
    int startTrancation = nIter + 1;
    bool flag_truncation = false;
    auto slotV = [&](int idx) -> DevBuf& { return ctx->slot(20 + 3 * (size_t)idx); };
    auto slotE = [&](int idx) -> DevBuf& { return ctx->slot(21 + 3 * (size_t)idx); };
    auto slotS = [&](int idx) -> DevBuf& { return ctx->slot(22 + 3 * (size_t)idx); };
    double* dThermo = nullptr;
    if (out && out->thermo) {
        DevBuf& bT = ctx->scratch.b[39];
        NRG_TRY(bT.ensure(sizeof(double) * 3 * (size_t)nIt));
        dThermo = bT.as<double>();
    }

    // the pinned eigenvalue buffer of the early path, sized once for the run: no iteration
    // keeps more than max(nOps * nb0, 1.2 N_keep) states (postprocess.F90:79-126), so no
    // iteration has more than nOps times that (capped at 4M values, 32 MB: a run that
    // effectively never truncates grows the buffer as it goes instead)
    if (ctx->early_evals) {
        const long long keep = std::max<long long>((long long)M.nOps * in->numberOfBasis,
                                                   (long long)(M.truncation * 1.2) + 1);
        NRG_TRY(ctx->h_evals.ensure(sizeof(double) * (size_t)std::min(keep * M.nOps, 1LL << 22)));
    }
    // ---- forward sweep ----
    // per-state bookkeeping on the device unless the operations change the quantum numbers
    // alike (NRG_HOST_TABLES=1 keeps all of it on the host; NRG_CHECK_TABLES=1 compares the
    // device's tables with the host's at every iteration)
    const bool dev_tables = ctx->device_tables && !env_flag("NRG_HOST_TABLES") && ops_change_qn_distinctly(M);
    const bool check_tables = dev_tables && env_flag("NRG_CHECK_TABLES");
    const bool flow_out = out && out->flow && out->flowStride > 0;
    const bool fdm_req = spectrum && in->temperature > 0.0;
    TruncTables TT;
    for (int it = first; it <= nIter; ++it) {
        const int idx = it - first;
        IterRec& R = recs[idx];
        Sectors& S = ctx->iter_sectors[idx];
        if (dev_tables && idx > 0) {   // from the previous iteration's sectors and kept counts
            std::vector<RowRun> runs;
            NRG_TRY(S.plan(M, ctx->iter_sectors[idx - 1], recs[idx - 1].kept, &runs));
            NRG_TRY(rows_device(ctx, S, runs));
            if (check_tables) NRG_TRY(check_device_rows(ctx, M, it, ctx->iter_sectors[idx - 1], recs[idx - 1].kept, S));
        } else {
            std::vector<int> rec, si;
            prepare_basis_host(M, bo, nb_old, &rec, &si);
            NRG_TRY(S.build((int)(si.size() / rs), si.data(), nb_old * M.nOps, rec.data(), nVar, M.nOps));
            NRG_TRY(S.upload(ctx));   // counted in ctx->h2d by the upload
        }
        const int nb = S.nb;
        const int nsub = S.nsub;
        const bool truncate = it != M.first && it != M.nIter && nb > M.truncation;   // postprocess.F90:79-81
        if (dev_tables) {
            TT.P = TruncParams();
            TT.P.nb = nb;
            TT.P.nsub = nsub;
            TT.P.truncate = truncate ? 1 : 0;
            TT.P.ntrunc = M.truncation;
            TT.P.limit = (int)(M.truncation * 1.2);
            NRG_TRY(TT.prepare(ctx, S));
        }
        // the host needs the energies themselves for the last iteration (ground states,
        // density-matrix seed), the full-density-matrix weights and the energy flow
        const bool need_E = !dev_tables || it == nIter || fdm_req || flow_out || check_tables;
        DevBuf& bV = slotV(idx);
        DevBuf& bE = slotE(idx);
        NRG_TRY(bV.ensure(sizeof(double) * (size_t)S.sizeV));
        NRG_TRY(bE.ensure(sizeof(double) * (size_t)nb));
        // the call returns with the shifted eigenvalues (or the device truncation's kept
        // counts) on the host while the eigenvectors are still being formed: the next
        // iteration's tables are built meanwhile, and every later launch on the stream is
        // ordered after them
        DiagOut dout;
        DiagPost post;
        post.early = ctx->early_evals;
        post.trunc = dev_tables ? &TT : nullptr;
        if (ctx->early_evals && need_E) {
            NRG_TRY(ctx->h_evals.ensure(sizeof(double) * (size_t)nb));
            post.h_E = ctx->h_evals.as<double>();
        }
        NRG_TRY(diag_device(ctx, it, S, dEold, nb_old, dIMold, bV.as<double>(), bE.as<double>(), &dout, &post));
        if (need_E) {
            if (ctx->early_evals) {
                R.Esec.assign(ctx->h_evals.as<double>(), ctx->h_evals.as<double>() + nb);
            } else {
                R.Esec.resize(nb);
                NRG_CUDA_TRY(cudaMemcpyAsync(R.Esec.data(), bE.p, sizeof(double) * nb, cudaMemcpyDeviceToHost, st));
                NRG_CUDA_TRY(cudaStreamSynchronize(st));
                ctx->d2h += (long long)sizeof(double) * nb;
            }
        }
        if (out && out->thermo) NRG_TRY(run_thermo(ctx, S, bE.as<double>(), dThermo + 3 * (size_t)idx));
        if (out && out->groundStateEnergy) out->groundStateEnergy[idx] = dout.groundStateEnergy;
        R.emin = dout.emin;
        int nbk = 0;
        std::vector<int> bo_new;
        std::vector<double> Eold_next;
        if (dev_tables) {
            NRG_TRY(TT.result(&R.kept, &nbk));
            if (truncate && startTrancation > it) {   // postprocess.F90:83-86
                startTrancation = it;
                flag_truncation = true;
            }
            std::vector<int> order;   // the kept rows in index order (flow, check)
            if (flow_out || check_tables) {
                for (int s = 0; s < nsub; ++s)
                    for (int t = 0; t < R.kept[s]; ++t) order.push_back(S.start[s] + t);
            }
            if (check_tables) {
                std::vector<int> ho;
                int st2 = nIter + 1;
                bool fl2 = false;
                const int nbk_h = truncate_host(M, it, R.Esec, &ho, &st2, &fl2);
                ho.resize(nbk_h);
                if (nbk_h != nbk || ho != order) {
                    nrg_set_error_message("iteration %d: the device truncation kept %d states, the host's %d", it, nbk,
                                          nbk_h);
                    return NRG_ERR_STATE;
                }
            }
            record_flow(out, idx, R.Esec, order, nbk);
        } else {
            std::vector<int> order;
            nbk = truncate_host(M, it, R.Esec, &order, &startTrancation, &flag_truncation);
            record_flow(out, idx, R.Esec, order, nbk);
            std::vector<int> rowSec(nb);
            for (int s = 0; s < nsub; ++s)
                for (int j = 0; j < S.dim[s]; ++j) rowSec[S.start[s] + j] = s;
            bo_new.assign((size_t)nb * rs, 0);
            Eold_next.resize(nbk);
            R.kept.assign(nsub, 0);
            for (int q = 0; q < nb; ++q) {
                const int row = order[q], s = rowSec[row];
                int* r = &bo_new[(size_t)q * rs];
                for (int v = 0; v < nVar; ++v) r[v] = S.qn[(size_t)s * nVar + v];
                r[nVar] = row - S.start[s] + 1;
                if (q < nbk) { Eold_next[q] = R.Esec[row]; R.kept[s]++; }
            }
        }
        R.nb_full = nb;
        R.nb_kept = nbk;
        if (out && out->kept) out->kept[idx] = nbk;
        if (out && out->numberOfBasisFull) out->numberOfBasisFull[idx] = nb;
        const double* dIMnew = dIMold;
        OpView imsNew = imsOld;
        if (it < nIter) {   // postprocess.F90:189-204
            DevBuf& bIM = ctx->slot(1 + ((idx + 1) & 1));
            NRG_TRY(bIM.ensure(sizeof(double) * (size_t)nbk * nbk * M.nCM));
            NRG_TRY(invmat_device(ctx, S, R.kept, bV.as<double>(), bIM.as<double>()));
            dIMnew = bIM.as<double>();
            if (spectrum) {
                NRG_TRY(invmat_spec_device(ctx, S, R.kept, bV.as<double>(), imsOld, nullptr, &imsTab[idx],
                                           &slotS(idx)));
                imsNew = OpView();
                imsNew.sp = &imsTab[idx];
            }
        }
        DevBuf& bEo = ctx->slot(3 + ((idx + 1) & 1));
        NRG_TRY(bEo.ensure(sizeof(double) * std::max(nbk, 1)));
        if (dev_tables) {
            NRG_TRY(TT.gather(ctx, bE.as<double>(), bEo.as<double>()));
        } else {
            NRG_TRY(h2d_async(ctx, bEo.p, Eold_next.data(), sizeof(double) * nbk));
            bo.swap(bo_new);
        }
        dEold = bEo.as<double>();
        dIMold = dIMnew;
        imsOld = imsNew;
        nb_old = nbk;
    }
    NRG_CUDA_TRY(cudaEventRecord(ev[1], st));

    const int nbin = M.numberOfBin();
    const size_t nw = (size_t)nbin * std::max(M.nMat, 1);
    DevBuf& bBins = ctx->slot(6);
    NRG_TRY(bBins.ensure(sizeof(double) * 2 * nw));
    double* dPos = bBins.as<double>();
    double* dNeg = dPos + nw;
    NRG_TRY(run_fill(ctx, dPos, (long long)(2 * nw), 0.0));

    // ---- full-density-matrix weights (temperature > 0; no reference counterpart) ----
    // P_s = d^(N_max - N) exp(-eps_s / T) / Z for the states discarded at shell N (all
    // states at the last shell), eps_s = scale(N) E_s + C_N with C_N - C_Nmax =
    // -sum_(N' > N) scale(N') min(H_N'): every shell on one energy scale measured from the
    // last shell's origin (small offsets keep eps / T precise at low T)
    const bool fdm = spectrum && in->temperature > 0.0;
    const int N0 = std::min(startTrancation, nIter);
    if (fdm && N0 <= first) {
        nrg_set_error_message("the full-density-matrix spectrum needs at least two NRG iterations");
        return NRG_ERR_UNSUPPORTED;
    }
    std::vector<long long> pOff(nIt, -1);
    std::vector<double> pShell(nIt, 0.0);
    DevBuf& bP = ctx->slot(11);
    if (fdm) {
        std::vector<double> C(nIt, 0.0);
        for (int N = nIter - 1; N >= first; --N) C[N - first] = C[N + 1 - first] - M.scale(N + 1) * recs[N + 1 - first].emin;
        const double T = in->temperature, lnd = std::log((double)M.nOps);
        long long tot = 0;
        for (int N = N0; N <= nIter; ++N) { pOff[N - first] = tot; tot += recs[N - first].nb_full; }
        std::vector<double> hP((size_t)std::max(tot, 1LL), 0.0);
        double vmax = -INFINITY;
        for (int pass = 0; pass < 2; ++pass) {
            double sum = 0.0;
            for (int N = N0; N <= nIter; ++N) {
                const IterRec& R = recs[N - first];
                const Sectors& S = ctx->iter_sectors[N - first];
                const double sc = M.scale(N);
                for (int s = 0; s < S.nsub; ++s)
                    for (int c = (N == nIter ? 0 : R.kept[s]); c < S.dim[s]; ++c) {
                        const double v = (nIter - N) * lnd - (sc * R.Esec[S.start[s] + c] + C[N - first]) / T;
                        if (pass == 0) vmax = std::max(vmax, v);
                        else hP[pOff[N - first] + S.start[s] + c] = v;
                        if (pass == 1) sum += std::exp(v - vmax);
                    }
            }
            if (pass == 1) {
                const double lnZ = vmax + std::log(sum);
                for (int N = N0; N <= nIter; ++N) {
                    const IterRec& R = recs[N - first];
                    const Sectors& S = ctx->iter_sectors[N - first];
                    double ps = 0.0;
                    for (int s = 0; s < S.nsub; ++s)
                        for (int c = (N == nIter ? 0 : R.kept[s]); c < S.dim[s]; ++c) {
                            double& p = hP[pOff[N - first] + S.start[s] + c];
                            p = std::exp(p - lnZ);
                            ps += p;
                        }
                    pShell[N - first] = ps;
                }
            }
        }
        NRG_TRY(bP.ensure(sizeof(double) * hP.size()));
        NRG_CUDA_TRY(cudaMemcpyAsync(bP.p, hP.data(), sizeof(double) * hP.size(), cudaMemcpyHostToDevice, st));
        NRG_CUDA_TRY(cudaStreamSynchronize(st));
        ctx->h2d += (long long)(sizeof(double) * hP.size());
    }
    auto dP = [&](int idx) -> const double* { return fdm ? bP.as<double>() + pOff[idx] : nullptr; };

    // ---- backward reduced density matrices (initializeReducedDensity, main.F90:188-201) ----
    DevBuf& bRdm = ctx->slot(5);
    const int last = nIter - first;
    if (spectrum && (flag_truncation || fdm)) {
        long long off = 0;
        for (int N = nIter; N >= N0; --N) {
            IterRec& R = recs[N - first];
            R.rdm_off.assign(R.kept.size(), -1);
            if (fdm && N == nIter) continue;   // the last shell is all discarded: weights only
            for (size_t s = 0; s < R.kept.size(); ++s)
                if (R.kept[s] > 0) { R.rdm_off[s] = off; off += (long long)R.kept[s] * R.kept[s]; }
        }
        NRG_TRY(bRdm.ensure(sizeof(double) * (size_t)std::max(off, 1LL)));
        NRG_TRY(run_fill(ctx, bRdm.as<double>(), off, 0.0));
        IterRec& RL = recs[last];
        const Sectors& SL = ctx->iter_sectors[last];
        int deg = 0;
        for (int i = 0; i < RL.nb_full; ++i) deg += RL.Esec[i] < 1.0e-8;
        const double inv = 1.0 / (double)deg;
        for (int s = 0; s < SL.nsub && !fdm; ++s)
            for (int p = 0; p < RL.kept[s]; ++p)
                if (RL.Esec[SL.start[s] + p] < 1.0e-8) {
                    NRG_TRY(h2d_async(ctx, bRdm.as<double>() + RL.rdm_off[s] + (long long)p * RL.kept[s] + p, &inv,
                                      sizeof(double)));
                    ctx->h2d += sizeof(double);
                }
        DevBuf& bTr = ctx->slot(7);
        NRG_TRY(bTr.ensure(sizeof(double) * (size_t)(nIter + 2)));
        for (int N = nIter - 1; N >= N0; --N) {
            IterView P, C;
            const int ip = N - first, ic = N + 1 - first;
            P.S = &ctx->iter_sectors[ip]; P.kept = recs[ip].kept; P.d_V = slotV(ip).as<double>();
            P.d_rdm = bRdm.as<double>(); P.rdm_off = recs[ip].rdm_off;
            C.S = &ctx->iter_sectors[ic]; C.kept = recs[ic].kept; C.d_V = slotV(ic).as<double>();
            C.d_rdm = bRdm.as<double>(); C.rdm_off = recs[ic].rdm_off;
            if (fdm) {
                C.d_P = dP(ic);
                if (N + 1 == nIter) C.kept.assign(C.kept.size(), 0);
            }
            NRG_TRY(rdm_step_device(ctx, P, C, bRdm.as<double>(), bTr.as<double>() + N));
        }
        if (out && out->rdmTrace) {
            std::vector<double> tr(nIter + 1, NAN);
            NRG_CUDA_TRY(cudaMemcpyAsync(tr.data(), bTr.p, sizeof(double) * (nIter + 1), cudaMemcpyDeviceToHost, st));
            NRG_CUDA_TRY(cudaStreamSynchronize(st));
            ctx->d2h += (long long)sizeof(double) * (nIter + 1);
            double done = 0.0;   // FDM: weight discarded up to and including shell N
            for (int N = 0; N <= nIter; ++N) {
                if (fdm && N >= N0) done += pShell[N - first];
                const bool has = (N >= (fdm ? N0 : startTrancation)) && N < nIter;
                out->rdmTrace[N] = has ? tr[N] + (fdm ? done : 0.0) : NAN;
            }
        }
    }
    NRG_CUDA_TRY(cudaEventRecord(ev[2], st));

    // ---- full-density-matrix spectrum (temperature > 0) ----
    if (fdm) {
        DevBuf& bTot = ctx->slot(10);
        NRG_TRY(bTot.ensure(sizeof(double) * 4 * M.nMat));
        for (int N = N0; N <= nIter; ++N) {
            const int idx = N - first;
            IterView V;
            V.S = &ctx->iter_sectors[idx]; V.kept = recs[idx].kept; V.d_V = slotV(idx).as<double>();
            V.d_Esec = slotE(idx).as<double>(); V.nb_kept = recs[idx].nb_kept;
            V.d_rdm = bRdm.as<double>(); V.rdm_off = recs[idx].rdm_off; V.d_P = dP(idx);
            OpView prev;
            prev.sp = &imsTab[idx - 1];
            NRG_TRY(spike_fdm_device(ctx, N, V, prev, N == nIter, dPos, dNeg, bTot.as<double>()));
        }
    }
    // ---- CFS spectrum (main.F90:204-224) ----
    if (spectrum && !fdm) {
        DevBuf& bTmp = ctx->slot(8);
        DevBuf& bTot = ctx->slot(10);
        NRG_TRY(bTmp.ensure(sizeof(double) * 2 * nw));
        NRG_TRY(bTot.ensure(sizeof(double) * 4 * M.nMat));
        for (int N = startTrancation; N <= nIter; ++N) {
            const int idx = N - first;
            IterView V;
            V.S = &ctx->iter_sectors[idx]; V.kept = recs[idx].kept; V.d_V = slotV(idx).as<double>();
            V.d_Esec = slotE(idx).as<double>(); V.nb_kept = recs[idx].nb_kept;
            V.d_rdm = bRdm.as<double>(); V.rdm_off = recs[idx].rdm_off;
            OpView prev;
            prev.sp = &imsTab[idx - 1];
            if (N == nIter) {
                std::vector<int> gs;
                const Sectors& S = *V.S;
                for (int s = 0; s < S.nsub; ++s)
                    for (int p = 0; p < S.dim[s]; ++p)
                        if (recs[idx].Esec[S.start[s] + p] < 1.0e-8) gs.push_back(s);
                NRG_TRY(spike_t0_device(ctx, N, V, gs, prev, dPos, dNeg));
            } else {
                double* tPos = bTmp.as<double>();
                double* tNeg = tPos + nw;
                NRG_TRY(run_fill(ctx, tPos, (long long)(2 * nw), 0.0));
                NRG_TRY(spike_cfs_device(ctx, N, V, prev, bRdm.as<double>(), tPos, tNeg, bTot.as<double>()));
                NRG_TRY(run_add(ctx, dPos, tPos, (long long)(2 * nw)));
            }
        }
    }
    NRG_CUDA_TRY(cudaEventRecord(ev[3], st));
    NRG_CUDA_TRY(cudaStreamSynchronize(st));
    NRG_TRY(flush_profile_timers(ctx));
    NRG_TRY(check_device_status(ctx));
    if (dThermo) {
        NRG_CUDA_TRY(cudaMemcpy(out->thermo, dThermo, sizeof(double) * 3 * (size_t)nIt, cudaMemcpyDeviceToHost));
        ctx->d2h += (long long)sizeof(double) * 3 * nIt;
    }
    if (out) {
        out->numberOfBin = nbin;
        out->startTrancation = startTrancation;
        if (spectrum && out->binnedSpikePositive && out->binnedSpikeNegative && out->binCapacity >= (int64_t)(2 * nw)) {
            write_bins(M, out, nbin, dPos, dNeg, true);
            ctx->d2h += (long long)(2 * nw * sizeof(double));
        }
        if (out->finalEigenvalue) {
            const IterRec& RL = recs[last];
            for (int i = 0; i < out->finalCapacity && i < RL.nb_full; ++i) out->finalEigenvalue[i] = RL.Esec[i];
        }
    }
    return NRG_OK;
}

// ------------------------------------------------------------------------------------
// host drop-in data flow: the Fortran caller's view
// ------------------------------------------------------------------------------------
struct HostRestore {
    std::vector<double> E;
    const double* V = nullptr;     // eigenvector blocks of the iteration (a pinned module array)
    const double* ims = nullptr;   // invariant matrices for the spectrum (pinned)
    long long nV = 0;
    std::vector<int> bo, bi, si;
    int nb = 0, nb_full = 0, nsub = 0;
};

// host slots of the host-array driver: the module arrays a Fortran caller keeps
// allocated (invariant matrices ping-pong, one eigenvector and one spectrum-matrix array
// per iteration for the restore stock, the full stock of eigenvectors)
constexpr size_t kHostIM = 0, kHostFV = 2, kHostRDM = 3, kHostV = 16, kHostIMS = 16 + 4096;

// one step of the CFS loop (cfsSpectrumCalculation, module.F90:1683-1706) through the
// drop-in spike entry points, from the restore stock of iteration N and N-1
int cfs_step_drop_in(nrg_context* ctx, int N, const std::vector<RestoreView>& its, int nb0, const double* ims0,
                     const std::vector<int>& fsi, const std::vector<int>& map, const double* rdm, long long nrdm,
                     double* binPos, double* binNeg, double* tot) {
    const Model& M = ctx->model;
    const RestoreView& R = its[N - M.first];
    const bool has_prev = N > M.first;
    nrg_spike_io sio;
    std::memset(&sio, 0, sizeof(sio));
    sio.numberOfSubspace = R.nsub; sio.subspaceInfo = R.si; sio.numberOfBasis = R.nb;
    sio.numberOfBasisFull = R.nb_full; sio.basis_input = R.bi; sio.basis_output = R.bo;
    sio.eigenvalue = R.E; sio.eigenvector = R.V; sio.sizeOfEigenvector = (int64_t)R.nV;
    sio.numberOfBasis_old = has_prev ? its[N - 1 - M.first].nb : nb0;
    sio.invariant_matrix_spectrum = has_prev ? its[N - 1 - M.first].ims : ims0;
    sio.fullSubspaceInfo = fsi.data(); sio.mapFullSubspaceInfo = map.data();
    sio.elementNumFullSubspace = (int32_t)(fsi.size() / (M.nVar + 6)); sio.reducedDensityMatrix = rdm;
    sio.sizeOfReducedDensity = (int64_t)nrdm; sio.numberOfBin = M.numberOfBin();
    sio.binnedSpikePositive = binPos; sio.binnedSpikeNegative = binNeg;
    sio.total_sum = tot;
    if (N == M.nIter) return nrg_spike_zero_temperature(ctx, N, &sio);
    return nrg_spike_cfs(ctx, N, &sio);
}

// the energy column of the bins (main.F90:142-157); the weights start at zero
void bin_energies(const Model& M, int nbin, std::vector<double>& pos, std::vector<double>& neg) {
    const size_t nw = (size_t)nbin * M.nMat;
    pos.assign(2 * nw, 0.0);
    neg.assign(2 * nw, 0.0);
    for (int m = 0; m < M.nMat; ++m)
        for (int i = 0; i < nbin; ++i) {
            const double e = std::pow(10.0, -15.0 + double(i) / 1000.0);
            pos[(size_t)m * nbin + i] = e;
            neg[(size_t)m * nbin + i] = -e;
        }
}

// loadRestart (module.F90:1787-1890) and the CFS loop of main.F90:204-224 from the
// file's iteration on: the NRG sweep and the density matrices are skipped, the file is
// rewritten before every later step when save is set
int resume_drop_in(nrg_context* ctx, nrg_run_output* out, cudaEvent_t* ev, const char* path, bool save) {
    const Model& M = ctx->model;
    const int nbin = M.numberOfBin(), first = M.first, nIter = M.nIter, nIt = nIter - first + 1;
    const size_t nw = (size_t)nbin * M.nMat;
    RestartData D;
    NRG_TRY(restart_load(path, M, nbin, &D));
    NRG_CUDA_TRY(cudaEventRecord(ev[1], ctx->stream));
    NRG_CUDA_TRY(cudaEventRecord(ev[2], ctx->stream));
    std::vector<double> tot(4 * M.nMat);
    const long long nfsi = (long long)(D.fsi.size() / (M.nVar + 6));
    for (int N = D.iteration; N <= nIter; ++N) {
        if (save && N > D.iteration) {
            int32_t hami[20];
            std::memcpy(hami, D.hami, sizeof(hami));
            hami[9] = D.its[N - 1 - first].nb;   // hami%numberOfBasis after getRestore(N-1)
            NRG_TRY(restart_save(path, M, N, hami, D.its, D.nb0, D.ims0.data(), D.rdm.data(), (long long)D.rdm.size(),
                                 D.fsi.data(), nfsi, D.map.data(), D.binPos.data(), D.binNeg.data(), nbin));
        }
        NRG_TRY(cfs_step_drop_in(ctx, N, D.its, D.nb0, D.ims0.data(), D.fsi, D.map, D.rdm.data(),
                                 (long long)D.rdm.size(), D.binPos.data(), D.binNeg.data(), tot.data()));
    }
    NRG_CUDA_TRY(cudaEventRecord(ev[3], ctx->stream));
    NRG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (out) {
        out->numberOfBin = nbin;
        out->startTrancation = D.hami[kHamiStartTrancation];
        if (out->binnedSpikePositive && out->binnedSpikeNegative && out->binCapacity >= (int64_t)(2 * nw))
            write_bins(M, out, nbin, D.binPos.data() + nw, D.binNeg.data() + nw, false);
        for (int x = 0; x < nIt; ++x) {   // what the file keeps of the sweep
            if (out->kept) out->kept[x] = D.its[x].nb;
            if (out->numberOfBasisFull) out->numberOfBasisFull[x] = D.its[x].nb_full;
            if (out->groundStateEnergy) out->groundStateEnergy[x] = std::nan("");
            if (out->thermo)
                for (int k = 0; k < 3; ++k) out->thermo[3 * x + k] = std::nan("");
            if (out->flow && out->flowStride > 0)
                for (int q = 0; q < out->flowStride; ++q) out->flow[(size_t)x * out->flowStride + q] = std::nan("");
        }
        if (out->rdmTrace)
            for (int N = 0; N <= nIter; ++N) out->rdmTrace[N] = std::nan("");
        if (out->finalEigenvalue) {
            const RestoreView& RL = D.its[nIt - 1];
            for (int i = 0; i < out->finalCapacity && i < RL.nb_full; ++i) out->finalEigenvalue[i] = RL.E[i];
        }
    }
    return NRG_OK;
}

int run_drop_in(nrg_context* ctx, const nrg_run_input* in, nrg_run_output* out, cudaEvent_t* ev) {
    const Model& M = ctx->model;
    const bool save = in->save_restart != 0, load = in->load_restart != 0;
    const char* rpath = (in->restart_file && in->restart_file[0]) ? in->restart_file : "restart.dat";
    if ((save || load) && !(in->spectrum && M.nMat > 0)) {
        nrg_set_error_message("restart.dat belongs to the CFS spectrum phase: the run has no spectrum");
        return NRG_ERR_INVALID;
    }
    ctx->host_pageable = in->host_arrays_pageable != 0;
    if (load) return resume_drop_in(ctx, out, ev, rpath, save);
    // profiling: the replay's own host work = its wall clock less the entry calls' parts
    const auto wall0 = std::chrono::steady_clock::now();
    const double entries0 = ctx->entry_s[0] + ctx->entry_s[1] + ctx->entry_s[2];
    if (out && out->thermo)   // thermodynamics are the caller's part of postprocess here
        for (int k = 0; k < 3 * (M.nIter - M.first + 1); ++k) out->thermo[k] = std::nan("");
    const int nVar = M.nVar, rs = nVar + 3, rsf = nVar + 6, first = M.first, nIter = M.nIter;
    const int nIt = nIter - first + 1;
    const bool spectrum = in->spectrum && M.nMat > 0;
    int nb_old = in->numberOfBasis;
    const int nb0 = in->numberOfBasis;
    const double* ims0 = in->invariant_matrix_spectrum;   // invariant_matrix_spectrum_initial
    if (nIt > (int)(kHostIMS - kHostV)) return NRG_ERR_TOO_LARGE;
    std::vector<int> bo(in->basis_output, in->basis_output + (size_t)nb_old * rs);
    std::vector<double> E(in->eigenvalue, in->eigenvalue + nb_old);
    double* IM = nullptr;
    const double* IMS = nullptr;
    {
        const size_t nim = (size_t)nb_old * nb_old * M.nCM;
        HostBuf& h = ctx->hslot(kHostIM);
        NRG_TRY(h.ensure(sizeof(double) * std::max<size_t>(nim, 1)));
        std::memcpy(h.p, in->invariant_matrix, sizeof(double) * nim);
        IM = h.as<double>();
        if (spectrum) {
            const size_t nis = (size_t)nb_old * nb_old * M.nMat;
            HostBuf& g = ctx->hslot(kHostIMS + nIt);
            NRG_TRY(g.ensure(sizeof(double) * std::max<size_t>(nis, 1)));
            std::memcpy(g.p, in->invariant_matrix_spectrum, sizeof(double) * nis);
            IMS = g.as<double>();
        }
    }
    std::vector<HostRestore> rest(nIt);
    int startTrancation = nIter + 1;
    bool flag_truncation = false;
    // the "full" stock (postprocess.F90:221-374)
    std::vector<int> fsi, fbi, fbo, map(nIter + 2, 0);
    std::vector<double> fE;
    HostBuf& hFV = ctx->hslot(kHostFV);
    long long nFV = 0;
    // postprocess.F90's copy of the kept eigenvector columns into the full stock runs on a
    // host thread beside the next routine calls; it is joined before the stock grows and
    // before the density matrices read it (and on every way out of this function)
    struct Joiner {
        std::thread t;
        void join() { if (t.joinable()) t.join(); }
        ~Joiner() { join(); }
    } stock_copy;
    long long pointFBI = 1, pointFBO = 1, pointFS = 1, pointFV = 1, sizeRDM = 0;
    for (int it = first; it <= nIter; ++it) {
        const int idx = it - first;
        std::vector<int> bi, si;
        if (prepare_basis_host(M, bo, nb_old, &bi, &si) - 1 > 0x7fffffffLL) {
            nrg_set_error_message("drop-in replay: iteration %d has more eigenvector entries than the 32-bit "
                                  "count_eigenvector of subspaceInfo holds", it);
            return NRG_ERR_TOO_LARGE;
        }
        const int nb = nb_old * M.nOps;
        const int nsub = (int)(si.size() / rs);
        long long sizeV = 0;
        for (int s = 0; s < nsub; ++s) sizeV += (long long)si[(size_t)s * rs + nVar] * si[(size_t)s * rs + nVar];
        std::vector<double> Enew(nb);
        HostBuf& hV = ctx->hslot(kHostV + idx);
        NRG_TRY(hV.ensure(sizeof(double) * (size_t)std::max(sizeV, 1LL)));
        double* Vnew = hV.as<double>();
        std::vector<int> bo_sec((size_t)nb * rs);
        double gse = 0.0;
        nrg_diagonalization_io dio;
        dio.numberOfSubspace = nsub; dio.subspaceInfo = si.data(); dio.numberOfBasis = nb;
        dio.basis_input = bi.data(); dio.numberOfBasis_old = nb_old; dio.eigenvalue_old = E.data();
        dio.invariant_matrix = IM; dio.eigenvalue = Enew.data(); dio.eigenvector = Vnew;
        dio.sizeOfEigenvector = sizeV; dio.basis_output = bo_sec.data(); dio.groundStateEnergy = &gse;
        NRG_TRY(nrg_diagonalization(ctx, it, &dio));
        if (out && out->groundStateEnergy) out->groundStateEnergy[idx] = gse;
        std::vector<int> order;
        const int nbk = truncate_host(M, it, Enew, &order, &startTrancation, &flag_truncation);
        record_flow(out, idx, Enew, order, nbk);
        std::vector<int> bo_re((size_t)nb * rs);
        std::vector<double> E_re(nb);
        for (int q = 0; q < nb; ++q) {
            std::memcpy(&bo_re[(size_t)q * rs], &bo_sec[(size_t)order[q] * rs], sizeof(int) * rs);
            E_re[q] = Enew[order[q]];
        }
        if (out && out->kept) out->kept[idx] = nbk;
        if (out && out->numberOfBasisFull) out->numberOfBasisFull[idx] = nb;
        double* IMn = nullptr;
        double* IMSn = nullptr;
        if (it < nIter) {
            HostBuf& h = ctx->hslot(kHostIM + ((idx + 1) & 1));
            NRG_TRY(h.ensure(sizeof(double) * std::max<size_t>((size_t)nbk * nbk * M.nCM, 1)));
            IMn = h.as<double>();
            nrg_invariant_matrix_io iio;
            iio.numberOfSubspace = nsub; iio.subspaceInfo = si.data(); iio.numberOfBasisFull = nb;
            iio.basis_input = bi.data(); iio.numberOfBasis = nbk; iio.basis_output = bo_re.data();
            iio.eigenvector = Vnew; iio.sizeOfEigenvector = sizeV; iio.numberOfBasis_old = nb_old;
            iio.invariant_matrix_spectrum_old = nullptr; iio.invariant_matrix = IMn;
            NRG_TRY(nrg_invariant_matrix_dgemm(ctx, it, &iio));
            if (spectrum) {
                HostBuf& g = ctx->hslot(kHostIMS + idx);
                NRG_TRY(g.ensure(sizeof(double) * std::max<size_t>((size_t)nbk * nbk * M.nMat, 1)));
                IMSn = g.as<double>();
                iio.invariant_matrix_spectrum_old = IMS;
                iio.invariant_matrix = IMSn;
                NRG_TRY(nrg_invariant_matrix_for_spectrum_dgemm(ctx, it, &iio));
            }
        }
        if (spectrum) {
            HostRestore& R = rest[idx];
            R.E = E_re; R.V = Vnew; R.nV = sizeV; R.bo = bo_re; R.bi = bi; R.si = si; R.nb = nbk; R.nb_full = nb;
            R.nsub = nsub;
            if (it < nIter) R.ims = IMSn;
            if (it >= startTrancation) {
                map[it + 1] = (int)pointFS;
                fbo.insert(fbo.end(), bo_re.begin(), bo_re.begin() + (size_t)nbk * rs);
                fE.insert(fE.end(), E_re.begin(), E_re.begin() + nbk);
                fbi.insert(fbi.end(), bi.begin(), bi.end());
                std::vector<int> kcount, kfirst;
                kept_in_sectors(si, nsub, bo_re, nbk, nVar, &kcount, &kfirst);
                long long add = 0;
                for (int s = 0; s < nsub; ++s) add += (long long)si[(size_t)s * rs + nVar] * kcount[s];
                stock_copy.join();
                NRG_TRY(hFV.ensure(sizeof(double) * (size_t)std::max(nFV + add, 1LL), true));
                struct Run { double* dst; const double* src; size_t n; };
                std::vector<Run> runs;
                for (int s = 0; s < nsub; ++s) {
                    const int k = kcount[s], first_out = kfirst[s];
                    if (k == 0) continue;
                    const int d = si[(size_t)s * rs + nVar];
                    for (int v = 0; v < nVar; ++v) fsi.push_back(si[(size_t)s * rs + v]);
                    fsi.push_back(d);
                    fsi.push_back(k);
                    fsi.push_back((int)pointFV);
                    fsi.push_back((int)(pointFBI + si[(size_t)s * rs + nVar + 2] - 1));
                    fsi.push_back((int)(pointFBO + first_out));
                    fsi.push_back(0);
                    sizeRDM += (long long)k * k;
                    const long long c0 = (long long)si[(size_t)s * rs + nVar + 1] - 1;
                    runs.push_back({hFV.as<double>() + nFV, Vnew + c0, (size_t)d * k});
                    nFV += (long long)d * k;
                    pointFV += (long long)d * k;
                    ++pointFS;
                }
                stock_copy.t = std::thread([runs = std::move(runs)]() {
                    for (const Run& r : runs) std::memcpy(r.dst, r.src, sizeof(double) * r.n);
                });
                pointFBI += nb;
                pointFBO += nbk;
            }
        }
        E.swap(E_re);
        bo.swap(bo_re);
        IM = IMn;
        IMS = IMSn;
        nb_old = nbk;
    }
    NRG_CUDA_TRY(cudaEventRecord(ev[1], ctx->stream));
    const int nbin = M.numberOfBin();
    const size_t nw = (size_t)nbin * std::max(M.nMat, 1);
    std::vector<double> binPos, binNeg;
    bin_energies(M, nbin, binPos, binNeg);
    stock_copy.join();
    double* rdm = nullptr;   // reducedDensityMatrix, a module array like the others
    long long nrdm = 0;
    const int elementNum = (int)(pointFS - 1);
    if (spectrum && flag_truncation) {
        // initializeReducedDensity.F90:32-78
        int deg = 0;
        for (int i = 0; i < nb_old; ++i) deg += E[i] < 1.0e-8;
        const double pf = (double)deg;
        HostBuf& hR = ctx->hslot(kHostRDM);
        NRG_TRY(hR.ensure(sizeof(double) * (size_t)std::max(sizeRDM, 1LL)));
        rdm = hR.as<double>();
        nrdm = sizeRDM;
        std::memset(rdm, 0, sizeof(double) * (size_t)nrdm);
        const int r0 = map[nIter + 1] - 1;
        int point = 1;
        for (int j = r0; j < elementNum; ++j) {
            int* f = &fsi[(size_t)j * rsf];
            f[nVar + 5] = point;
            const int k = f[nVar + 1];
            for (int a = 0; a < k; ++a)
                if (fE[(size_t)f[nVar + 4] - 1 + a] < 1.0e-8) rdm[(size_t)point - 1 + (size_t)a * k + a] = 1.0 / pf;
            point += k * k;
        }
        nrg_reduced_density_io rio;
        rio.numberOfIteration = nIter; rio.startTrancation = startTrancation; rio.mapFullSubspaceInfo = map.data();
        rio.elementNumFullSubspace = elementNum; rio.fullSubspaceInfo = fsi.data();
        rio.fullBasisInput = fbi.data(); rio.numFullBasisInput = (int64_t)(fbi.size() / rs);
        rio.fullBasisOutput = fbo.data(); rio.numFullBasisOutput = (int64_t)(fbo.size() / rs);
        rio.fullEigenvector = hFV.as<double>(); rio.numFullEigenvector = (int64_t)nFV;
        rio.reducedDensityMatrix = rdm; rio.sizeOfReducedDensity = (int64_t)nrdm;
        rio.pointReducedDensity = &point;
        std::vector<double> tr(std::max(nIter - startTrancation, 1));
        rio.trace = tr.data();
        NRG_TRY(nrg_reduced_density_matrix(ctx, &rio));
        if (out && out->rdmTrace)
            for (int N = 0; N <= nIter; ++N)
                out->rdmTrace[N] = (N >= startTrancation && N < nIter) ? tr[nIter - 1 - N] : NAN;
    }
    NRG_CUDA_TRY(cudaEventRecord(ev[2], ctx->stream));
    if (spectrum) {
        std::vector<RestoreView> views(nIt);
        for (int x = 0; x < nIt; ++x) {
            const HostRestore& R = rest[x];
            RestoreView& v = views[x];
            v.si = R.si.data(); v.bi = R.bi.data(); v.bo = R.bo.data(); v.E = R.E.data(); v.V = R.V;
            v.ims = R.ims; v.nV = R.nV; v.nb = R.nb; v.nb_full = R.nb_full; v.nsub = R.nsub;
        }
        std::vector<double> tot(4 * M.nMat);
        for (int N = startTrancation; N <= nIter; ++N) {
            if (save) {   // main.F90:216-220: before every step, overwriting the file
                int32_t hami[20];
                const int nbh = N == startTrancation ? rest[nIt - 1].nb : rest[N - 1 - first].nb;
                restart_hami(M, nbh, startTrancation, flag_truncation, hami);
                NRG_TRY(restart_save(rpath, M, N, hami, views, nb0, ims0, rdm, nrdm,
                                     fsi.data(), (long long)elementNum, map.data(), binPos.data(), binNeg.data(),
                                     nbin));
            }
            NRG_TRY(cfs_step_drop_in(ctx, N, views, nb0, ims0, fsi, map, rdm, nrdm, binPos.data(), binNeg.data(),
                                     tot.data()));
        }
    }
    NRG_CUDA_TRY(cudaEventRecord(ev[3], ctx->stream));
    NRG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (ctx->profiling)
        ctx->replay_host_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - wall0).count() -
                              (ctx->entry_s[0] + ctx->entry_s[1] + ctx->entry_s[2] - entries0);
    if (out) {
        out->numberOfBin = nbin;
        out->startTrancation = startTrancation;
        if (spectrum && out->binnedSpikePositive && out->binnedSpikeNegative && out->binCapacity >= (int64_t)(2 * nw))
            write_bins(M, out, nbin, binPos.data() + nw, binNeg.data() + nw, false);
        if (out->finalEigenvalue) {
            // the last iteration keeps every state in sector order (no truncation)
            for (int i = 0; i < out->finalCapacity && i < (int)E.size(); ++i) out->finalEigenvalue[i] = E[i];
        }
    }
    return NRG_OK;
}

int run_one(nrg_context* ctx, const nrg_run_input* in, nrg_run_output* out);

}  // namespace

extern "C" int nrg_prepare_basis(int32_t numberOfVariation, int32_t numberOfOperation, int32_t numberOfChain,
                                 const int32_t* operation, int32_t numberOfBasis_old, const int32_t* basis_output,
                                 int32_t* basis_input, int32_t* subspaceInfo, int32_t subspaceCapacity,
                                 int32_t* numberOfSubspace) {
    const int nVar = numberOfVariation, nOps = numberOfOperation, rs = nVar + 3;
    if (nVar < 1 || nOps < 1 || numberOfChain < 0 || numberOfBasis_old < 0 || subspaceCapacity < 0 || !operation ||
        !numberOfSubspace || (numberOfBasis_old > 0 && (!basis_output || !basis_input || !subspaceInfo))) {
        nrg_set_error_message("nrg_prepare_basis: inconsistent sizes or NULL arrays");
        return NRG_ERR_INVALID;
    }
    if ((long long)numberOfBasis_old * nOps > 0x7fffffffLL) {
        nrg_set_error_message("nrg_prepare_basis: %d x %d states exceed the 32-bit basis index", numberOfBasis_old,
                              nOps);
        return NRG_ERR_TOO_LARGE;
    }
    Model M;
    M.nVar = nVar;
    M.nOps = nOps;
    M.nChain = numberOfChain;
    M.operation.assign(operation, operation + (size_t)nOps * (nVar + numberOfChain));
    std::vector<int> bo(basis_output, basis_output + (size_t)numberOfBasis_old * rs), rec, si;
    const long long ce_end = prepare_basis_host(M, bo, numberOfBasis_old, &rec, &si);
    const int nsub = (int)(si.size() / rs);
    *numberOfSubspace = nsub;
    if (ce_end - 1 > 0x7fffffffLL) {
        // the last sector's block would start beyond 2^31 - 1 or end there
        nrg_set_error_message("nrg_prepare_basis: the eigenvector blocks hold %lld entries, more than the 32-bit "
                              "count_eigenvector of subspaceInfo addresses", ce_end - 1);
        return NRG_ERR_TOO_LARGE;
    }
    if (nsub > subspaceCapacity) {
        nrg_set_error_message("nrg_prepare_basis: %d sectors, subspaceInfo holds %d", nsub, subspaceCapacity);
        return NRG_ERR_INVALID;
    }
    std::memcpy(basis_input, rec.data(), sizeof(int) * rec.size());
    std::memcpy(subspaceInfo, si.data(), sizeof(int) * si.size());
    return NRG_OK;
}

extern "C" int nrg_truncate(int32_t iteration, int32_t indexOfFirstIteration, int32_t numberOfIteration,
                            int32_t truncation, int32_t numberOfVariation, int32_t numberOfBasis, double* eigenvalue,
                            int32_t* basis_output, int32_t* numberOfBasis_kept, int32_t* startTrancation,
                            int32_t* flag_truncation) {
    if (numberOfBasis < 0 || truncation < 1 || numberOfVariation < 1 || !numberOfBasis_kept || !startTrancation ||
        !flag_truncation || (numberOfBasis > 0 && !eigenvalue)) {
        nrg_set_error_message("nrg_truncate: inconsistent sizes or NULL arrays");
        return NRG_ERR_INVALID;
    }
    Model M;
    M.first = indexOfFirstIteration;
    M.nIter = numberOfIteration;
    M.truncation = truncation;
    M.nVar = numberOfVariation;
    const int nb = numberOfBasis, rs = numberOfVariation + 3;
    std::vector<double> E(eigenvalue, eigenvalue + nb);
    std::vector<int> order;
    int st = *startTrancation;
    bool fl = *flag_truncation != 0;
    const int nbk = truncate_host(M, iteration, E, &order, &st, &fl);
    for (int q = 0; q < nb; ++q) eigenvalue[q] = E[order[q]];
    if (basis_output) {
        std::vector<int> bo(basis_output, basis_output + (size_t)nb * rs);
        for (int q = 0; q < nb; ++q)
            std::memcpy(basis_output + (size_t)q * rs, &bo[(size_t)order[q] * rs], sizeof(int) * rs);
    }
    *numberOfBasis_kept = nbk;
    *startTrancation = st;
    *flag_truncation = fl ? 1 : 0;
    return NRG_OK;
}

extern "C" int nrg_run(nrg_context* ctx, const nrg_run_input* in, nrg_run_output* out) {
    return run_one(ctx, in, out);
}

extern "C" int nrg_run_batch(nrg_context* const* ctxs, const nrg_run_input* in, nrg_run_output* out,
                             int32_t count, int32_t concurrency, int32_t flags, int32_t* statuses) {
    if (count < 0 || (count > 0 && (!ctxs || !in || !out))) {
        nrg_set_error_message("nrg_run_batch: NULL arrays or negative count");
        return NRG_ERR_INVALID;
    }
    for (int i = 0; i < count; ++i)
        for (int j = 0; j < i; ++j)
            if (ctxs[i] == ctxs[j]) {
                nrg_set_error_message("nrg_run_batch: instance %d repeats the context of instance %d", i, j);
                return NRG_ERR_INVALID;
            }
    const int nthr = std::max(1, std::min<int>(concurrency < 1 ? count : concurrency, count));
    std::vector<int> st(count, NRG_OK);
    std::atomic<int> next{0};
    std::mutex mu;
    int first_bad = -1;
    std::string first_msg;
    auto worker = [&]() {
        for (;;) {
            const int i = next.fetch_add(1);
            if (i >= count) return;
            nrg_context* c = ctxs[i];
            int rc = NRG_OK;
            cudaStream_t own = nullptr;
            if (!c) {
                nrg_set_error_message("nrg_run_batch: instance %d has no context", i);
                rc = NRG_ERR_INVALID;
            } else if (cudaSetDevice(c->device) != cudaSuccess) {
                cudaGetLastError();
                nrg_set_error_message("nrg_run_batch: cudaSetDevice(%d) failed", c->device);
                rc = NRG_ERR_CUDA;
            } else if (!c->stream) {
                // the legacy default stream would serialise the instances
                if (cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking) != cudaSuccess) {
                    cudaGetLastError();
                    nrg_set_error_message("nrg_run_batch: stream creation failed");
                    rc = NRG_ERR_CUDA;
                } else {
                    c->stream = own;
                }
            }
            if (rc == NRG_OK) {
                const bool early = c->early_evals;
                c->early_evals = early && nthr == 1;
                rc = run_one(c, in + i, out + i);
                c->early_evals = early;
            }
            if (c && (flags & NRG_BATCH_RELEASE)) {
                const int rr = nrg_context_release_storage(c);
                if (rc == NRG_OK) rc = rr;
            }
            if (own) {
                cudaStreamSynchronize(own);
                c->stream = nullptr;
                cudaStreamDestroy(own);
            }
            st[i] = rc;
            if (rc != NRG_OK) {
                std::lock_guard<std::mutex> lk(mu);
                if (first_bad < 0 || i < first_bad) {
                    first_bad = i;
                    first_msg = nrg_last_error();
                }
            }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nthr; ++t) pool.emplace_back(worker);
    worker();
    for (auto& t : pool) t.join();
    if (statuses)
        for (int i = 0; i < count; ++i) statuses[i] = st[i];
    if (first_bad >= 0) {
        nrg_set_error_message("instance %d: %s", first_bad, first_msg.c_str());
        return st[first_bad];
    }
    return NRG_OK;
}

namespace {
int run_one(nrg_context* ctx, const nrg_run_input* in, nrg_run_output* out) {
    if (!ctx || !in) return NRG_ERR_INVALID;
    if (!ctx->model.set) { nrg_set_error_message("nrg_context_set_model has not been called"); return NRG_ERR_STATE; }
    NRG_CUDA_TRY(cudaSetDevice(ctx->device));
    cudaEvent_t ev[4];
    for (auto& e : ev) NRG_CUDA_TRY(cudaEventCreate(&e));
    NRG_CUDA_TRY(cudaEventRecord(ev[0], ctx->stream));
    const int rc = in->host_drop_in ? run_drop_in(ctx, in, out, ev) : run_device(ctx, in, out, ev);
    if (rc == NRG_OK && out && out->phaseSeconds) {
        float a = 0, b = 0, c = 0;
        cudaEventElapsedTime(&a, ev[0], ev[1]);
        cudaEventElapsedTime(&b, ev[1], ev[2]);
        cudaEventElapsedTime(&c, ev[2], ev[3]);
        out->phaseSeconds[0] = a * 1e-3;
        out->phaseSeconds[1] = b * 1e-3;
        out->phaseSeconds[2] = c * 1e-3;
        out->phaseSeconds[3] = (a + b + c) * 1e-3;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    return rc;
}
}  // namespace
