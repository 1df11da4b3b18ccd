// Internal structures shared by the C ABI (capi.cu), the device-resident driver
// (driver.cu) and the kernels.
#pragma once
#include "common.cuh"

#include <string>
#include <vector>
#include <map>
#include <deque>
#include <mutex>
#include <unordered_map>

namespace nrg {

// ------------------------------------------------------------------------------------
// grow-only device buffer
// ------------------------------------------------------------------------------------
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    int ensure(size_t want);
    void release();
    template <class T> T* as() const { return static_cast<T*>(p); }
};

// grow-only pinned host buffer (module arrays of the host-array driver); keep = true
// preserves the contents when the buffer grows
struct HostBuf {
    void* p = nullptr;
    size_t bytes = 0;
    bool pageable = false;         // the next allocation: plain malloc instead of page-locked
    bool alloc_pageable = false;   // how p was allocated
    int ensure(size_t want, bool keep = false);
    void release();
    template <class T> T* as() const { return static_cast<T*>(p); }
};

// ------------------------------------------------------------------------------------
// model tables (host copies + device copies + derived lookup tables)
// ------------------------------------------------------------------------------------
struct Model {
    bool set = false;
    int nIter = 0, nChain = 0, nVar = 0, cb[4] = {0, 0, 0, 0}, nMat = 0, nCM = 0, nCoef = 0,
        nOps = 0, nBCS = 0, first = 0, flag_spectrum = 0, flag_BCS = 0;
    double D = 1, z = 1, Lambda = 2;
    int scalingType = 1, truncation = 0;
    std::vector<int> operation;          // (nOps, nVar+nChain) col-major
    std::vector<double> chain_diag;      // (nIter+2, nChain)
    std::vector<double> chain_nond;      // (nIter+2-first, nChain)
    std::vector<double> chain_bcs;       // (nIter+2, nChain)
    std::vector<double> cspec;           // (nMat, nOps)
    std::vector<int> cons_diff, pos_op, neg_op;  // (nMat, nVar)
    // outcome of the coefficient scans, per (op_i, op_j) (diagonalization.F90:195-224)
    std::vector<int> dflag, dtype, dch, dswp, bflag, bch;
    std::vector<double> dcoef;
    // invariantMatrixDGEMM.F90:248-254, per (op_l, op_r, type)
    std::vector<int> imflag;
    std::vector<double> imcoef;
    // device copies
    DevBuf d_operation, d_dflag, d_dtype, d_dch, d_dswp, d_bflag, d_bch, d_dcoef, d_imflag, d_imcoef;

    double scale(int N) const;
    double cd(int N, int c) const { return chain_diag[(size_t)N + (size_t)c * (nIter + 2)]; }
    double cn(int N, int c) const { return chain_nond[(size_t)(N - first) + (size_t)c * (nIter + 2 - first)]; }
    double cbcs(int N, int c) const { return chain_bcs.empty() ? 0.0 : chain_bcs[(size_t)N + (size_t)c * (nIter + 2)]; }
    int op(int j, int col) const { return operation[(size_t)j + (size_t)col * nOps]; }
    int numberOfBin() const;
};

// ------------------------------------------------------------------------------------
// per-iteration sector tables built from subspaceInfo + basis_input
// ------------------------------------------------------------------------------------
// one run of rows of the next iteration's basis: the kept states of one old sector
// combined with one operation (tables.cu)
struct RowRun {
    int row0;       // first row (0-based) of basis_input
    int len;        // rows: the old sector's kept states
    int ref0;       // 0-based reference of the first row (kept states before the old sector)
    int op;         // 0-based operation
    int sec;        // new sector
    int sec_start;  // its first row
    int lst0;       // offset of the (sector, operation) row list
};

struct Sectors {
    int nsub = 0, nb = 0, nVar = 0, nOps = 0;
    std::vector<int> qn;        // nsub*nVar
    std::vector<int> dim, start;        // start: 0-based row of basis_input
    std::vector<long long> ce;          // 0-based offset of the eigenvector block
    long long sizeV = 0;
    std::vector<int> rowOp, rowRef, rowVar;   // per row (0-based op / ref, 1-based var)
    // rows of sector s with local operation a, ordered by variation: local row indices
    std::vector<int> lst, lstOff;       // lstOff: nsub*nOps + 1
    std::vector<int> refBase;           // nsub*nOps: 0-based reference of the first listed row
    // device copies
    DevBuf d_bi, d_lst, d_lstOff;
    int build(int nsub, const int* si, int nb, const int* bi, int nVar, int nOps);
    int upload(nrg_context* ctx);
    // The table prepareBasis builds for the next iteration, from this iteration's sectors
    // and kept counts alone (tables.cu; models whose operations change the quantum numbers
    // in pairwise different ways).  Fills the sector-level fields; the per-row records and
    // row lists are written on the device by rows_device from the returned runs.
    int plan(const Model& M, const Sectors& prev, const std::vector<int>& kept_prev, std::vector<RowRun>* runs);
    void index_qn();                    // rebuilds qnHash from qn
    int find(const int* q) const;       // findSubspace: first sector with these qn, or -1
    std::vector<int> qnHash;            // open-addressing index of the sectors by qn (find)
    static unsigned long long hash_qn(const int* q, int nVar);
    int cnt(int s, int a) const { return lstOff[s * nOps + a + 1] - lstOff[s * nOps + a]; }
};

// ------------------------------------------------------------------------------------
// the context
// ------------------------------------------------------------------------------------
struct Scratch {
    DevBuf b[48];
};

}  // namespace nrg

namespace nrg {
// per-device choice of the grouped GEMM's tile shape (ggemm.cu)
struct GemmTuner {
    static constexpr int kTunedVariants = 4, kSamples = 2;
    struct Entry {
        double ms_per_gflop[kTunedVariants] = {0.0, 0.0, 0.0, 0.0};
        int samples[kTunedVariants] = {0, 0, 0, 0};
        int inflight[kTunedVariants] = {0, 0, 0, 0};
    };
    struct Pending {
        unsigned key;
        int variant;
        cudaEvent_t a, b;
        double gflop;
    };
    std::mutex mu;
    std::unordered_map<unsigned, Entry> table;
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> free_events;
    int pick(unsigned key);
    void collect(bool wait);
    int event(cudaEvent_t* e);
};
}  // namespace nrg

struct nrg_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    nrg::Model model;
    nrg::Scratch scratch;
    nrg::DevBuf d_status;
    long long launches = 0;
    // measurement counters (nrg_context_get_stats)
    bool profiling = false;
    long long syev_launches = 0;
    double syev_ms = 0.0, syev_flops = 0.0;
    long long h2d = 0, d2h = 0;
    long long tri_launches = 0;
    double tri_ms = 0.0, tri_flops = 0.0, tri_bytes = 0.0;
    double entry_s[3] = {0.0, 0.0, 0.0};   // drop-in entries: staging in, device, out
    long long entry_calls = 0;
    double replay_host_s = 0.0;
    // driver-owned persistent storage, reused across runs
    std::deque<nrg::DevBuf> store;
    std::vector<nrg::Sectors> iter_sectors;
    // pinned staging ring for small host-to-device uploads (tables, index lists): a copy
    // from pageable memory would wait for the stream to drain first
    struct StageChunk { size_t begin, end; cudaEvent_t ev; };
    char* stage_host = nullptr;
    size_t stage_cap = 0, stage_head = 0;
    std::deque<StageChunk> stage_inflight;
    std::vector<cudaEvent_t> event_pool;
    // second stream: the one-block-per-sector eigensolver of the small sectors runs beside
    // the large-sector pipeline (fork / join events on the caller's stream)
    cudaStream_t aux = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    // third stream: the large sectors below the largest size class run their pipeline
    // beside the largest sectors' (whose tridiagonalisation sets the critical path)
    cudaStream_t aux2 = nullptr, aux_hi = nullptr;   // aux_hi: greatest priority, the largest sectors
    cudaEvent_t ev_join2 = nullptr, ev_join_hi = nullptr;
    // tridiagonalisation timers (profiling on), read once the eigensolver has joined so
    // that timing does not stall the launch queue
    struct PendingTimer { cudaEvent_t a, b; double flops, bytes; };
    std::vector<PendingTimer> pending_tri;
    std::vector<PendingTimer> pending_syev;   // eigensolver windows (flops only)
    // early eigenvalues (device-resident sweep): each large-sector group records its
    // event once the divide and conquer has written the eigenvalues; the caller's stream
    // shifts them and copies them to pinned host memory (ev_evals_host) before it waits
    // for the back-transformations, so the host bookkeeping of the next iteration runs
    // while they finish
    cudaEvent_t ev_evals_hi = nullptr, ev_evals2 = nullptr, ev_evals_host = nullptr;
    cudaStream_t aux_copy = nullptr;        // eigenvector blocks to the host as their groups end
    cudaEvent_t ev_copied = nullptr;
    // measured policy: the early path gains ~6 % for an instance that has the device to
    // itself and loses ~10 % with eight instances in flight (their work already fills
    // the host gap), so nrg_run_batch turns it off when it runs instances side by side
    bool early_evals = true;
    nrg::HostBuf h_small;   // pinned: the shift's minimum and E(1), the status word
    nrg::HostBuf h_evals;   // pinned: the shifted eigenvalues of the current iteration
    nrg::HostBuf h_kept;    // pinned: the device truncation's kept counts
    bool device_tables = true;   // per-state bookkeeping of nrg_run on the device (tables.cu)
    nrg::DevBuf& slot(size_t i) {
        if (store.size() <= i) store.resize(i + 1);
        return store[i];
    }
    // device copies of the drop-in entries' sector tables (basis, index lists), kept
    // between calls: an entry borrows a set and gives it back, so once the buffers have
    // grown its calls allocate and free nothing (a free would also wait for the device)
    struct TableBufs { nrg::DevBuf bi, lst, off; };
    std::deque<TableBufs> table_pool;
    TableBufs& table_slot(size_t i) {
        if (table_pool.size() <= i) table_pool.resize(i + 1);
        return table_pool[i];
    }
    // host module arrays of the host-array driver, reused across runs: page-locked, or
    // pageable like a Fortran allocatable when host_pageable is set
    std::deque<nrg::HostBuf> host_store;
    bool host_pageable = false;
    // page-locked staging of the runs a routine reads from a caller's pageable array
    std::deque<nrg::HostBuf> seg_stage;
    nrg::HostBuf& seg_slot(size_t i) {
        if (seg_stage.size() <= i) seg_stage.resize(i + 1);
        return seg_stage[i];
    }
    nrg::HostBuf& hslot(size_t i) {
        if (host_store.size() <= i) host_store.resize(i + 1);
        host_store[i].pageable = host_pageable;
        return host_store[i];
    }
    ~nrg_context();
};

namespace nrg {

// a strided run of a host array: count runs of len doubles from element off, ld apart
struct HostSeg {
    long long off;
    int len, count;
};
// copies the listed runs of src (device-accessible pinned host memory) to the same
// positions of dst, reading them over the host link from a kernel; ld is the stride
// between the runs of one segment.  packed: src holds the runs one after another (in
// segment order) instead of at their positions.
int run_gather_segs(nrg_context* ctx, const double* src, double* dst, long long ld,
                    const std::vector<HostSeg>& segs, long long* bytes, bool packed = false);

// raises a kernel's dynamic shared-memory limit on the current device to at least bytes
// and never lowers it: the attribute belongs to the kernel, not to a stream, and host
// threads running independent contexts launch the same kernels with different sizes
int raise_smem_limit(const void* func, size_t bytes);

// stream-ordered upload of a small host array through the pinned staging ring (the host
// array may be reused as soon as the call returns)
int h2d_async(nrg_context* ctx, void* dst, const void* src, size_t bytes);

// ---- grouped gather GEMM -------------------------------------------------------------
struct GemmProblem {
    int M, N, K;
    int tiles;              // filled by the launcher
    double alpha, beta;
    // A(i,k) = A[ri(i)*a_si + ki(k)*a_sk], ri = a_ri ? a_ri[i] : i, ki = a_ki ? a_ki[k] : k
    const double* A; long long a_si, a_sk; const int* a_ri; const int* a_ki;
    const double* B; long long b_sk, b_sj; const int* b_ki; const int* b_ji;
    // C(i,j) = C[ri(i)*c_si + ji(j)*c_sj]
    double* C; long long c_si, c_sj; const int* c_ri; const int* c_ji;
    // when set, N and K are read from device memory (N = min(N, *dyn_nk), K = *dyn_nk);
    // the launch is sized for the static N
    const int* dyn_nk;
};
int launch_ggemm(nrg_context* ctx, std::vector<GemmProblem>& probs, int scratch_slot);



// eigensolver for sectors of order > 128 across the whole GPU (eig_large.cu); the
// descriptors use a_off / e_off / n only
// (scratch slots slot_base .. slot_base + 6; on ctx->stream)
// evals_ready (optional) is recorded on ctx->stream once the eigenvalues are in d_E,
// before the back-transformation
int syev_large(nrg_context* ctx, const std::vector<SyevSector>& secs, double* d_V, double* d_E, int slot_base,
               cudaEvent_t evals_ready = nullptr);
constexpr int kLargeSector = 128;

// ---- kernels (kernels.cu) ------------------------------------------------------------
int run_assemble(nrg_context* ctx, int iteration, const Sectors& S, const SyevSector* d_secs,
                 const long long* d_colPrefix, const int* d_secStart, int nsec, long long ncols,
                 const double* d_Eold, int nb_old, const double* d_IMold, double* d_V);
// the shift of the eigenvalues (E -= min E, E <= 1e-12 -> 0; min and E(1) to
// d_min_and_gs) and the chop of the eigenvectors (|V| < 1e-14 -> 0), on ctx->stream
int run_eig_shift(nrg_context* ctx, double* d_E, int nb, double* d_min_and_gs);
int run_eig_chop(nrg_context* ctx, long long sizeV, double* d_V, cudaStream_t st = nullptr);   // null: ctx->stream

struct ImGatherProb {
    long long t_off;    // T (dL x kR) col-major
    long long vR_off;   // V_R block
    int L, R, t, dL, dR, kR, startL;
};
int run_im_gather(nrg_context* ctx, const Sectors& S, std::vector<ImGatherProb>& probs,
                  const double* d_V, double* d_T);

struct SpikeProb {
    long long s_off, y_off;   // S, Y (kk x nl) col-major in the workspace (y_off < 0: T=0)
    long long ek_off, el_off; // offsets into the energy array (k states, l states)
    int kk, nl, m, toPos, lstride;  // lstride: 1 for consecutive l energies, 0 for a fixed one
    double sgn, cE, scale, invpf;
    // full-density-matrix mode: spikes of the sign of this job's bins only; weights
    // P (same offsets as the energies) on both sides; k_is_y: k holds the extra particle
    int fdm, k_is_y;
};
int run_spikes(nrg_context* ctx, std::vector<SpikeProb>& probs, const double* d_work,
               const double* d_E, int nbin, int nMat, double* d_binPos, double* d_binNeg,
               double* d_tot, const double* d_P = nullptr);
int run_fill(nrg_context* ctx, double* p, long long n, double v);
// dst[i + j n] = V[rows[i] + (c0 + j) ld] * P[j]: gathered rows of a column range scaled by
// per-column weights, for many blocks in one launch
struct ScaledGather {
    long long dst, v, rows, p;
    int n, nc, ld, c0;
};
int run_scaled_gather(nrg_context* ctx, const std::vector<ScaledGather>& jobs, double* dst, const double* V,
                      const int* rows, const double* P);
// betabar of module.F90:652, a default-real literal (single precision 0.8 widened)
constexpr double kBetabar = (double)0.8f;
// calcThermo (module.F90:1931-1982) of one iteration: d_out[0..2] = Cn, Sn, Xn
int run_thermo(nrg_context* ctx, const Sectors& S, const double* d_E, double* d_out);
// log-Gaussian broadening of binned spikes onto the frequencies d_omega: d_A[m*nw + k]
int run_broaden(nrg_context* ctx, const double* d_bins, int nbin, int nMat, double b, const double* d_omega,
                int nw, double* d_A);
int run_add(nrg_context* ctx, double* dst, const double* src, long long n);
int run_sum_bins(nrg_context* ctx, const double* bins, int nbin, int nMat, double* out);
int run_trace(nrg_context* ctx, const double* rdm, const long long* d_offs, const int* d_dims,
              int nblk, double* out);
int run_gather_rows(nrg_context* ctx, double* dst, long long dst_ld, const double* src,
                    long long src_ld, const int* d_rows, int nrows, int ncols);

// ---- internal routines shared by the ABI and the driver (routines.cu) ------------------
struct DiagOut {
    double groundStateEnergy = 0.0;   // eigenvalue(1) before the shift (the reference's)
    double emin = 0.0;                // the minimum subtracted by the shift
};
// diagonalization for one iteration; d_Eold/d_IMold/d_V/d_E are device pointers.
// With h_E (pinned host, nb doubles) the call returns as soon as the shifted eigenvalues
// are in h_E: the eigenvectors are still being formed on the device, ordered before
// any later work on ctx->stream.
// Work diag_device does for the device-resident run right after the eigenvalue shift, on
// the caller's stream.  early: return once the shifted eigenvalues' minimum, the status
// word, h_E and the truncation's counts have reached the host, before the eigenvectors are
// complete (later launches on the stream still follow them); h_E (early only): pinned copy
// of the shifted eigenvalues, or null.  Without early the call returns with the stream
// drained.
struct DiagPost {
    bool early = false;
    double* h_E = nullptr;
    struct TruncTables* trunc = nullptr;   // device truncation launched after the shift
    // Without early: the caller's page-locked eigenvector array (the drop-in's module
    // array), or null.  When the largest sectors run on their own stream, the blocks of the
    // other sectors are chopped and copied there as soon as their groups end, on a copy
    // stream, while the largest sectors are still being reduced; theirs follow.  The call
    // returns with every block in h_V (the caller then copies nothing).
    double* h_V = nullptr;
    bool copied_V = false;                 // out: h_V holds the eigenvectors
};
int diag_device(nrg_context* ctx, int iteration, Sectors& S, const double* d_Eold, int nb_old,
                const double* d_IMold, double* d_V, double* d_E, DiagOut* out, DiagPost* post = nullptr);

// ---- device bookkeeping of the device-resident run (tables.cu) ----
struct TruncParams {
    int nb = 0, nsub = 0;
    int truncate = 0;              // the rule of postprocess.F90:79-126 applies
    int ntrunc = 0;                // param%truncation (N_keep)
    int limit = 0;                 // int(N_keep * truncationLimitScale)
    double thr = 0.000001;         // truncationThreshold (module.F90:629)
    double step = 0.001;           // the cut-back step (postprocess.F90:109)
    long long max_steps = 1LL << 24;   // bound of the cut-back loop (the reference has none)
};
struct TruncTables {
    TruncParams P;
    int nsub = 0;
    int* d_secTab = nullptr;       // start, dimension per sector
    int* d_out = nullptr;          // kept total, status, kept per sector
    int* d_koff = nullptr;         // kept states before each sector
    double* d_ecut = nullptr;
    int* h_out = nullptr;          // pinned copy of d_out
    int prepare(nrg_context* ctx, const Sectors& S);
    int launch(nrg_context* ctx, const double* d_E);    // kernel + copy of the counts to h_out
    int result(std::vector<int>* kept, int* nb_kept) const;   // after h_out has arrived
    int gather(nrg_context* ctx, const double* d_E, double* d_Enext) const;
};
int rows_device(nrg_context* ctx, Sectors& S, const std::vector<RowRun>& runs);
bool ops_change_qn_distinctly(const Model& M);
// reads the profiling timers of completed eigensolver windows into the counters
int flush_profile_timers(nrg_context* ctx);

// ---- restart.dat of the CFS phase (restart.cu; module.F90:1710-1890) -------------------
// one iteration of the restore stock as getRestore hands it to the spike routines
struct RestoreView {
    const int* si = nullptr;     // subspaceInfo [nsub*(nVar+3)]
    const int* bi = nullptr;     // basis_input [nb_full*(nVar+3)]
    const int* bo = nullptr;     // basis_output after the truncation reorder
    const double* E = nullptr;   // eigenvalue [nb_full], same order as bo
    const double* V = nullptr;   // eigenvector blocks [nV]
    const double* ims = nullptr; // d† matrices of the kept states (nb, nb, nMat); none at the last iteration
    long long nV = 0;
    int nb = 0, nb_full = 0, nsub = 0;
};
// words of HamiltonianInfo_type (module.F90:722-760) read back by the drop-in replay
constexpr int kHamiStartTrancation = 17, kHamiFlagTruncation = 18;
struct RestartData {
    int32_t iteration = 0;
    int32_t hami[20];
    int nb0 = 0;
    std::vector<int32_t> restoreInfo, si, bi, bo, fsi, map;
    std::vector<double> ims, ims0, E, V, rdm, binPos, binNeg;
    std::vector<RestoreView> its;   // first .. nIter, pointing into the arrays above
};
void restart_hami(const Model& M, int numberOfBasis, int startTrancation, bool flag_truncation, int32_t hami[20]);
// its: iterations first .. nIter; map: mapFullSubspaceInfo(-1:nIter); bins (nbin*nMat, 2)
int restart_save(const char* path, const Model& M, int iteration, const int32_t hami[20],
                 const std::vector<RestoreView>& its, int nb0, const double* ims0, const double* rdm, long long nrdm,
                 const int* fsi, long long nfsi, const int* map, const double* binPos, const double* binNeg,
                 int nbin);
int restart_load(const char* path, const Model& M, int nbin, RestartData* D);

// kept counts per sector from the kept prefix of basis_output (invariantMatrixDGEMM.F90:84-100)
std::vector<int> kept_per_sector(const Sectors& S, int nb_kept, const int* basis_output_kept);

int invmat_device(nrg_context* ctx, const Sectors& S, const std::vector<int>& kept,
                  const double* d_V, double* d_IM);

// The d-dagger matrices <l| d^dagger_m |r> of the kept states of one iteration, stored as
// blocks: only the (sector L, sector R, m) blocks whose quantum numbers differ by the
// operator's (invariantMatrixForSpectrumDGEMM.F90:166-170) are kept, each column-major
// kept[R] x kept[L] (element (r, l) at off + r + l * kept[R]); the others are zero.
struct SparseBlocks {
    int nsub = 0, nMat = 0;
    std::vector<long long> kst;   // kept-state prefix per sector (nsub + 1)
    std::vector<int> kept;        // kept states per sector
    std::vector<long long> off;   // ((L * nsub) + R) * nMat + m -> offset, -1 when absent
    long long total = 0;          // doubles
    const double* data = nullptr;
    int sector_of(long long i) const;   // sector holding kept index i, or -1
};
// read access to a d-dagger matrix of the kept states of one iteration: dense
// (nb, nb, nMat) column-major as the reference stores it, or block-sparse
struct OpView {
    const double* dense = nullptr;
    long long nb = 0;
    const SparseBlocks* sp = nullptr;
    // element (r0, l0, m) of a cr x cl range and its strides along r and l; nullptr when
    // the range lies in an absent (zero) block; *bad when the range leaves the matrix or
    // crosses a block boundary
    const double* at(long long r0, long long l0, int m, long long cr, long long cl, long long* sr,
                     long long* sl, bool* bad) const;
};
// invariantMatrixForSpectrumDGEMM: the new matrix, dense into d_dense (nb_kept^2 x nMat) or,
// with d_dense null, block-sparse into *sp_out with its data in *sp_buf
int invmat_spec_device(nrg_context* ctx, const Sectors& S, const std::vector<int>& kept,
                       const double* d_V, const OpView& old, double* d_dense, SparseBlocks* sp_out,
                       DevBuf* sp_buf);

// rdm / spectrum inputs for one iteration (device resident)
struct IterView {
    const Sectors* S = nullptr;
    std::vector<int> kept;            // kept per sector
    const double* d_P = nullptr;      // full-density-matrix weights by state (sector order), or null
    const double* d_V = nullptr;      // all eigenvector blocks
    const double* d_Esec = nullptr;   // eigenvalues in sector order
    int nb_kept = 0;
    // reduced density blocks of the kept sectors (row-major k x k), device offsets
    const double* d_rdm = nullptr;
    std::vector<long long> rdm_off;   // per sector, -1 when the sector has no kept state
};
int rdm_step_device(nrg_context* ctx, const IterView& present, const IterView& child,
                    double* d_rdm, double* d_trace_out);
// blocks of the previous d-dagger matrix (nb_old x nb_old x nMat) the spike routines read:
// T = 0 jobs when gs_sectors is given, CFS jobs otherwise
std::vector<HostSeg> spike_ims_segs(const Model& M, const IterView& it, const std::vector<int>* gs_sectors,
                                    int nb_old);
int spike_cfs_device(nrg_context* ctx, int iteration, const IterView& it, const OpView& old,
                     const double* d_rdm, double* d_binPos, double* d_binNeg, double* d_tot);
int spike_t0_device(nrg_context* ctx, int iteration, const IterView& it,
                    const std::vector<int>& gs_sectors, const OpView& old,
                    double* d_binPos, double* d_binNeg);
// full-density-matrix spectrum of one shell: the kept-discarded terms (the CFS products,
// with the discarded states' weights added) and the discarded-discarded terms, each
// spike in the bins of the sign of its frequency; last: every state is discarded
int spike_fdm_device(nrg_context* ctx, int iteration, const IterView& it, const OpView& old,
                     bool last, double* d_binPos, double* d_binNeg, double* d_tot);

int check_device_status(nrg_context* ctx);

}  // namespace nrg
