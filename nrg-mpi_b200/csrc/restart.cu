// restart.dat of the CFS phase: saveRestart / loadRestart (module.F90:1710-1890).
//
// The file is Fortran unformatted stream output (access="stream": raw bytes, no record
// markers), little endian, default integers and logicals 4 bytes (gfortran: .true. = 1),
// reals 8 bytes.  A derived-type item is written as its components in order
// (HamiltonianInfo_type, module.F90:722-760: 20 four-byte words; type restore,
// module.F90:983-994: 10 integers).  Layout, in the order of saveRestart:
//   mode (MODE_RESTART_CFS = 1002), iteration, hami,
//   lbound, ubound, restoreInfo(:),
//   size, restore_subspaceInfo memory   (records of nVar+3 ints)
//   size, restore_basis_input memory    (records of nVar+3 ints)
//   size, restore_basis_output memory   (records of nVar+3 ints)
//   size, restore_invariant_matrix_spectrum(:)
//   dims 1..3, invariant_matrix_spectrum_initial(:,:,:)
//   size, restoreEigenvalue(:)
//   size, restoreEigenVector(:)
//   size, reducedDensityMatrix(:)
//   size, fullSubspaceInfo memory       (records of nVar+6 ints)
//   lbound, ubound, mapFullSubspaceInfo(:)
//   size, binnedSpikePositive(:,:)      (numberOfBin*nMat x 2, energies then weights)
//   size, binnedSpikeNegative(:,:)
// "size" of a record array counts records; of a real array, elements.
#include "internal.hpp"

#include <cstdio>
#include <cstring>
#include <limits>
#include <vector>

namespace nrg {

namespace {

constexpr int32_t kModeRestartCfs = 1002;   // module.F90:1720
constexpr int kRestoreFields = 10;          // type restore, module.F90:983-994

struct File {
    FILE* f = nullptr;
    ~File() {
        if (f) fclose(f);
    }
};

int put(FILE* f, const void* p, size_t bytes) {
    if (bytes && fwrite(p, 1, bytes, f) != bytes) {
        nrg_set_error_message("restart file: write failed");
        return NRG_ERR_INVALID;
    }
    return NRG_OK;
}
int put_i(FILE* f, long long v) {
    if (v < std::numeric_limits<int32_t>::min() || v > std::numeric_limits<int32_t>::max()) {
        nrg_set_error_message("restart file: %lld does not fit the file's 4-byte integers", v);
        return NRG_ERR_TOO_LARGE;
    }
    const int32_t x = (int32_t)v;
    return put(f, &x, 4);
}
int get(FILE* f, void* p, size_t bytes) {
    if (bytes && fread(p, 1, bytes, f) != bytes) {
        nrg_set_error_message("broken restart file: truncated");
        return NRG_ERR_INVALID;
    }
    return NRG_OK;
}
int get_i(FILE* f, int32_t* v) { return get(f, v, 4); }
int get_count(FILE* f, int32_t* v) {
    NRG_TRY(get_i(f, v));
    if (*v < 0) {
        nrg_set_error_message("broken restart file: negative size");
        return NRG_ERR_INVALID;
    }
    return NRG_OK;
}
// n elements read into v; a count read from the file is checked against the bytes the
// file still holds before anything is allocated, so a damaged count is reported as a
// broken file rather than failing an allocation
template <class T>
int get_vec(FILE* f, std::vector<T>& v, size_t n) {
    const long long here = ftello(f);
    long long end = -1;
    if (here >= 0 && fseeko(f, 0, SEEK_END) == 0) end = ftello(f);
    if (end < here || fseeko(f, here, SEEK_SET) != 0) {
        nrg_set_error_message("broken restart file: cannot seek");
        return NRG_ERR_INVALID;
    }
    if (n > (size_t)(end - here) / sizeof(T)) {
        nrg_set_error_message("broken restart file: truncated");
        return NRG_ERR_INVALID;
    }
    v.resize(n);
    return get(f, v.data(), sizeof(T) * n);
}

}  // namespace

void restart_hami(const Model& M, int numberOfBasis, int startTrancation, bool flag_truncation, int32_t hami[20]) {
    // HamiltonianInfo_type components in order (module.F90:722-760); the two the hot path
    // does not take (numberOfCoefficientImpurity, flag_local) hold their defaults
    int k = 0;
    hami[k++] = M.nIter;
    hami[k++] = M.nChain;
    hami[k++] = M.nVar;
    for (int i = 0; i < 4; ++i) hami[k++] = M.cb[i];
    hami[k++] = M.nMat;
    hami[k++] = M.nCM;
    hami[k++] = numberOfBasis;
    hami[k++] = M.nCoef;
    hami[k++] = 0;                  // numberOfCoefficientImpurity
    hami[k++] = M.nOps;
    hami[k++] = M.nBCS;
    hami[k++] = M.first;
    hami[k++] = M.flag_spectrum ? 1 : 0;
    hami[k++] = 0;                  // flag_local
    hami[k++] = startTrancation;
    hami[k++] = flag_truncation ? 1 : 0;
    hami[k++] = M.flag_BCS ? 1 : 0;
}

int restart_save(const char* path, const Model& M, int iteration, const int32_t hami[20],
                 const std::vector<RestoreView>& its, int nb0, const double* ims0, const double* rdm, long long nrdm,
                 const int* fsi, long long nfsi, const int* map, const double* binPos, const double* binNeg,
                 int nbin) {
    const int nIt = M.nIter - M.first + 1;
    if ((int)its.size() != nIt) {
        nrg_set_error_message("restart_save: %zu iterations for %d", its.size(), nIt);
        return NRG_ERR_INVALID;
    }
    const int rs = M.nVar + 3, rsf = M.nVar + 6;
    // restoreInfo(first:nIter+1) (initRestore / appendRestore, module.F90:1388-1567):
    // running starts; the last iteration stores no spectrum matrix and the extra entry
    // nIter+1 is never filled (written as zeros)
    std::vector<long long> ri((size_t)(nIt + 1) * kRestoreFields, 0);
    long long e0 = 1, v0 = 1, s0 = 1, m0 = 1, nsi = 0, nrec = 0, nims = 0, nE = 0, nV = 0;
    for (int x = 0; x < nIt; ++x) {
        const RestoreView& R = its[x];
        long long* r = &ri[(size_t)x * kRestoreFields];
        r[0] = e0; r[1] = R.nb_full;
        r[2] = v0; r[3] = R.nV;
        r[4] = s0; r[5] = R.nsub;
        r[6] = e0;
        const long long nm = (M.first + x < M.nIter) ? (long long)R.nb * R.nb * M.nMat : 0;
        r[7] = nm ? m0 : 0; r[8] = nm;
        r[9] = R.nb;
        e0 += R.nb_full; v0 += R.nV; s0 += R.nsub; m0 += nm;
        nsi += R.nsub; nrec += R.nb_full; nims += nm; nE += R.nb_full; nV += R.nV;
    }
    File F;
    F.f = fopen(path, "wb");
    if (!F.f) {
        nrg_set_error_message("cannot open restart file %s for writing", path);
        return NRG_ERR_INVALID;
    }
    FILE* f = F.f;
    NRG_TRY(put_i(f, kModeRestartCfs));
    NRG_TRY(put_i(f, iteration));
    NRG_TRY(put(f, hami, 4 * 20));
    NRG_TRY(put_i(f, M.first));
    NRG_TRY(put_i(f, M.nIter + 1));
    for (long long v : ri) NRG_TRY(put_i(f, v));
    NRG_TRY(put_i(f, nsi));
    for (const RestoreView& R : its) NRG_TRY(put(f, R.si, sizeof(int) * (size_t)R.nsub * rs));
    NRG_TRY(put_i(f, nrec));
    for (const RestoreView& R : its) NRG_TRY(put(f, R.bi, sizeof(int) * (size_t)R.nb_full * rs));
    NRG_TRY(put_i(f, nrec));
    for (const RestoreView& R : its) NRG_TRY(put(f, R.bo, sizeof(int) * (size_t)R.nb_full * rs));
    NRG_TRY(put_i(f, nims));
    for (int x = 0; x < nIt; ++x)
        if (M.first + x < M.nIter)
            NRG_TRY(put(f, its[x].ims, sizeof(double) * (size_t)its[x].nb * its[x].nb * M.nMat));
    NRG_TRY(put_i(f, nb0));
    NRG_TRY(put_i(f, nb0));
    NRG_TRY(put_i(f, M.nMat));
    NRG_TRY(put(f, ims0, sizeof(double) * (size_t)nb0 * nb0 * M.nMat));
    NRG_TRY(put_i(f, nE));
    for (const RestoreView& R : its) NRG_TRY(put(f, R.E, sizeof(double) * (size_t)R.nb_full));
    NRG_TRY(put_i(f, nV));
    for (const RestoreView& R : its) NRG_TRY(put(f, R.V, sizeof(double) * (size_t)R.nV));
    NRG_TRY(put_i(f, nrdm));
    NRG_TRY(put(f, rdm, sizeof(double) * (size_t)nrdm));
    NRG_TRY(put_i(f, nfsi));
    NRG_TRY(put(f, fsi, sizeof(int) * (size_t)nfsi * rsf));
    NRG_TRY(put_i(f, -1));
    NRG_TRY(put_i(f, M.nIter));
    NRG_TRY(put(f, map, sizeof(int) * (size_t)(M.nIter + 2)));
    const size_t nw = (size_t)nbin * M.nMat * 2;
    NRG_TRY(put_i(f, (long long)nw));
    NRG_TRY(put(f, binPos, sizeof(double) * nw));
    NRG_TRY(put_i(f, (long long)nw));
    NRG_TRY(put(f, binNeg, sizeof(double) * nw));
    if (fflush(f) != 0) {
        nrg_set_error_message("restart file: write failed");
        return NRG_ERR_INVALID;
    }
    return NRG_OK;
}

int restart_load(const char* path, const Model& M, int nbin, RestartData* D) {
    File F;
    F.f = fopen(path, "rb");
    if (!F.f) {   // loadRestart aborts with "restart file not found" (module.F90:1799-1805)
        nrg_set_error_message("restart file not found: %s", path);
        return NRG_ERR_INVALID;
    }
    FILE* f = F.f;
    int32_t mode = 0;
    NRG_TRY(get_i(f, &mode));
    if (mode != kModeRestartCfs) {   // module.F90:1811-1817
        nrg_set_error_message("broken restart file: mode %d", mode);
        return NRG_ERR_INVALID;
    }
    NRG_TRY(get_i(f, &D->iteration));
    NRG_TRY(get(f, D->hami, 4 * 20));
    const int32_t* h = D->hami;
    const bool same = h[0] == M.nIter && h[1] == M.nChain && h[2] == M.nVar && h[7] == M.nMat && h[8] == M.nCM &&
                      h[12] == M.nOps && h[14] == M.first;
    if (!same) {
        nrg_set_error_message("restart file %s belongs to another model (numberOfIteration %d, numberOfVariation %d, "
                              "numberOfOperation %d, indexOfFirstIteration %d)", path, h[0], h[2], h[12], h[14]);
        return NRG_ERR_INVALID;
    }
    const int rs = M.nVar + 3, rsf = M.nVar + 6, nIt = M.nIter - M.first + 1;
    int32_t lo = 0, hi = 0, n = 0;
    NRG_TRY(get_i(f, &lo));
    NRG_TRY(get_i(f, &hi));
    if (lo != M.first || hi < M.nIter || hi > M.nIter + 1) {
        nrg_set_error_message("broken restart file: restoreInfo(%d:%d)", lo, hi);
        return NRG_ERR_INVALID;
    }
    NRG_TRY(get_vec(f, D->restoreInfo, (size_t)(hi - lo + 1) * kRestoreFields));
    NRG_TRY(get_count(f, &n));
    NRG_TRY(get_vec(f, D->si, (size_t)n * rs));
    NRG_TRY(get_count(f, &n));
    NRG_TRY(get_vec(f, D->bi, (size_t)n * rs));
    NRG_TRY(get_count(f, &n));
    NRG_TRY(get_vec(f, D->bo, (size_t)n * rs));
    NRG_TRY(get_count(f, &n));
    NRG_TRY(get_vec(f, D->ims, (size_t)n));
    int32_t d1 = 0, d2 = 0, d3 = 0;
    NRG_TRY(get_count(f, &d1));
    NRG_TRY(get_count(f, &d2));
    NRG_TRY(get_count(f, &d3));
    if (d1 != d2 || d3 != M.nMat || d1 > (1 << 20)) {
        nrg_set_error_message("broken restart file: initial spectrum matrices (%d, %d, %d)", d1, d2, d3);
        return NRG_ERR_INVALID;
    }
    D->nb0 = d1;
    NRG_TRY(get_vec(f, D->ims0, (size_t)d1 * d2 * d3));
    NRG_TRY(get_count(f, &n));
    NRG_TRY(get_vec(f, D->E, (size_t)n));
    NRG_TRY(get_count(f, &n));
    NRG_TRY(get_vec(f, D->V, (size_t)n));
    NRG_TRY(get_count(f, &n));
    NRG_TRY(get_vec(f, D->rdm, (size_t)n));
    NRG_TRY(get_count(f, &n));
    NRG_TRY(get_vec(f, D->fsi, (size_t)n * rsf));
    NRG_TRY(get_i(f, &lo));
    NRG_TRY(get_i(f, &hi));
    if (lo != -1 || hi != M.nIter) {
        nrg_set_error_message("broken restart file: mapFullSubspaceInfo(%d:%d)", lo, hi);
        return NRG_ERR_INVALID;
    }
    NRG_TRY(get_vec(f, D->map, (size_t)(hi - lo + 1)));
    const size_t nw = (size_t)nbin * M.nMat * 2;
    for (std::vector<double>* b : {&D->binPos, &D->binNeg}) {
        NRG_TRY(get_count(f, &n));
        if ((size_t)n != nw) {
            nrg_set_error_message("restart file %s: %d bin entries, the model has %zu", path, n, nw);
            return NRG_ERR_INVALID;
        }
        NRG_TRY(get_vec(f, *b, nw));
    }
    // per-iteration views of the stock (getRestore, module.F90:1596-1660), bounds checked
    D->its.assign(nIt, RestoreView());
    for (int x = 0; x < nIt; ++x) {
        const int32_t* r = &D->restoreInfo[(size_t)x * kRestoreFields];
        RestoreView& R = D->its[x];
        R.nb_full = r[1];
        R.nV = r[3];
        R.nsub = r[5];
        R.nb = r[9];
        const long long e = (long long)r[0] - 1, v = (long long)r[2] - 1, s = (long long)r[4] - 1,
                        b = (long long)r[6] - 1, m = (long long)r[7] - 1;
        const bool last = M.first + x == M.nIter;
        const long long nm = last ? 0 : (long long)R.nb * R.nb * M.nMat;
        const bool ok = R.nb_full >= 0 && R.nV >= 0 && R.nsub >= 0 && R.nb >= 0 && R.nb <= R.nb_full && e >= 0 &&
                        e + R.nb_full <= (long long)D->E.size() && v >= 0 && v + R.nV <= (long long)D->V.size() &&
                        s >= 0 && (s + R.nsub) * rs <= (long long)D->si.size() && b >= 0 &&
                        (b + R.nb_full) * rs <= (long long)D->bi.size() &&
                        (b + R.nb_full) * rs <= (long long)D->bo.size() &&
                        (last || (r[8] == nm && m >= 0 && m + nm <= (long long)D->ims.size()));
        if (!ok) {
            nrg_set_error_message("broken restart file: restoreInfo(%d) out of range", M.first + x);
            return NRG_ERR_INVALID;
        }
        R.E = D->E.data() + e;
        R.V = D->V.data() + v;
        R.si = D->si.data() + s * rs;
        R.bi = D->bi.data() + b * rs;
        R.bo = D->bo.data() + b * rs;
        R.ims = last ? nullptr : D->ims.data() + m;
    }
    if (D->iteration < h[kHamiStartTrancation] || D->iteration > M.nIter) {
        nrg_set_error_message("restart file %s: iteration %d outside the CFS loop %d..%d", path, D->iteration,
                              h[kHamiStartTrancation], M.nIter);
        return NRG_ERR_INVALID;
    }
    return NRG_OK;
}

}  // namespace nrg
