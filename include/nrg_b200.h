/*
 * nrg_b200.h -- C ABI of the B200 NRG hot path.
 *
 * The reference (eminamitani/nrg-mpi, Fortran 90 + MPI + OpenMP + LAPACK/BLAS) keeps all
 * state in module globals and calls its hot routines without arguments.  Each entry point
 * below replaces one of those routines; its arguments are exactly the module arrays the
 * routine reads and writes (raw pointers, sizes, 1-based integer values inside the
 * packed records, Fortran column-major real arrays), so a Fortran caller binds them with
 * ISO_C_BINDING: a bind(C) interface block for the entries and records below, and
 * wrapper subroutines with the reference's names that pass the module arrays.
 *
 * Pointers may be host or device memory (CUDA unified addressing tells them apart).
 * Host arrays are copied to the device inside the call and results copied back before
 * the call returns, so the call is a drop-in for the synchronous Fortran routine.
 *
 * Packed integer records (module.F90):
 *   Basis_type            [basis(1:nVar), reference, variation, operation]   (:440-466)
 *   SubspaceInfo_type     [basis(1:nVar), dimension, count_eigenvector, start_input] (:167-194)
 *   FullSubspaceInfo_type [basis(1:nVar), dimension_before, dimension_after,
 *                          start_eigen, start_input, start_output, start_matrix] (:294-327)
 *
 * Every call returns an NRG_* status; nrg_last_error() describes the last failure.
 * There is no CPU fallback: without a usable CUDA device every compute call fails with
 * NRG_ERR_DEVICE.  The two host bookkeeping entries (nrg_prepare_basis, nrg_truncate)
 * are integer and sorting work that the reference also does on the host; they need no
 * device.
 */
#ifndef NRG_B200_H
#define NRG_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define NRG_API __attribute__((visibility("default")))
#else
#define NRG_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

enum {
    NRG_OK = 0,
    NRG_ERR_INVALID = 1,      /* an argument is inconsistent (sizes, indices, NULL)   */
    NRG_ERR_CUDA = 2,         /* a CUDA runtime call failed                          */
    NRG_ERR_NOMEM = 3,        /* device allocation failed                            */
    NRG_ERR_TOO_LARGE = 4,    /* a block exceeds a kernel's size plan                */
    NRG_ERR_DEVICE = 5,       /* no usable CUDA device                                */
    NRG_ERR_UNSUPPORTED = 6,  /* input outside what the kernels implement            */
    NRG_ERR_STATE = 7,        /* call sequence error (e.g. no model set)             */
    NRG_ERR_NUMERIC = 8,      /* a kernel flagged a numerical failure                */
    NRG_ERR_TIMEOUT = 9       /* a bounded device wait expired                       */
};

typedef struct nrg_context nrg_context;

/* Model-wide inputs: what setupHamiltonian, read_parameter and read_initial_basis fill
 * (module.F90:612-626, 722-760, 826-944; read_initial_basis.F90:27-204).  Chains are
 * passed already rescaled (read_initial_basis.F90:103-142). */
typedef struct nrg_model {
    int32_t numberOfIteration;
    int32_t numberOfChain;
    int32_t numberOfVariation;
    int32_t conservationBlock[4];            /* Fortran conservationBlock(2,2), col-major */
    int32_t numberOfMatrix;
    int32_t numberOfConductionMatrix;
    int32_t numberOfCoefficient;
    int32_t numberOfOperation;
    int32_t numberOfBCSCoefficient;
    int32_t indexOfFirstIteration;
    int32_t flag_spectrum;
    int32_t flag_BCS;
    double bandWidth;
    double ztrick;
    double Lambda;
    int32_t scalingType;
    int32_t truncation;
    const int32_t* operation;                         /* (nOps, nVar+nChain)          */
    const int32_t* coefficient_invariant_matrix_type; /* (nCoef, 3)                    */
    const double* coefficient_invariant_matrix;       /* (nCoef)                       */
    const int32_t* coefficient_diagonalization_type;  /* (nCoef, 4)                    */
    const double* coefficient_diagonalization;        /* (nCoef)                       */
    const double* chain_diagonal;                     /* (0:nIter+1, nChain)           */
    const double* chain_nondiagonal;                  /* (first:nIter+1, nChain)       */
    const double* chain_BCS;                          /* (0:nIter+1, nChain) or NULL   */
    const int32_t* coefficient_BCS;                   /* (nBCS, 3) or NULL             */
    const double* coefficient_invariant_matrix_spectrum; /* (nMat, nOps)               */
    const int32_t* conservation_difference_spectrum;  /* (nMat, nVar)                  */
    const int32_t* positiveSpectrumOperation;         /* (nMat, nVar)                  */
    const int32_t* negativeSpectrumOperation;         /* (nMat, nVar)                  */
} nrg_model;

/* ---- context ------------------------------------------------------------------------ */
NRG_API int nrg_context_create(nrg_context** ctx, int device);
NRG_API int nrg_context_destroy(nrg_context* ctx);
/* CUDA stream (cudaStream_t) the kernels are launched on; NULL = the default stream. */
NRG_API int nrg_context_set_stream(nrg_context* ctx, void* stream);
/* Copies the model tables into the context (setupHamiltonian + read_initial_basis). */
NRG_API int nrg_context_set_model(nrg_context* ctx, const nrg_model* model);
/* Number of kernels this library launched on the context since creation. */
NRG_API int64_t nrg_context_launch_count(const nrg_context* ctx);

/* Counters for measurement (no counterpart in the reference; it times phases with
 * count.f90).  Eigensolver times are taken with CUDA events around each batched launch
 * when profiling is on; its algorithmic flops are sum over sectors of (4/3 + 2) d^3. */
typedef struct nrg_stats {
    int64_t launches;        /* kernels launched                                      */
    int64_t syev_launches;   /* batched eigensolver launches                           */
    double syev_ms;          /* their summed device time (profiling on)               */
    double syev_flops;       /* algorithmic flops of those launches                   */
    int64_t h2d_bytes;       /* host-to-device bytes moved by the library             */
    int64_t d2h_bytes;       /* device-to-host bytes moved by the library             */
    int64_t tri_launches;    /* cluster tridiagonalisation launches (profiling on)    */
    double tri_ms;           /* their summed device time                              */
    double tri_flops;        /* their algorithmic flops, sum over sectors of 4/3 n^3  */
    double tri_bytes;        /* their algorithmic matrix reads, sum of 8 n^3 / 3      */
    /* drop-in entry points (profiling on: the stream is drained between the parts, so
     * the parts do not overlap), host wall-clock seconds summed over calls:            */
    double entry_in_s;       /* host tables, sector build, host-to-device staging     */
    double entry_compute_s;  /* the device work                                       */
    double entry_out_s;      /* device-to-host results, host-side output work         */
    int64_t entry_calls;     /* drop-in entry calls timed                             */
    double replay_host_s;    /* nrg_run's host drop-in replay: its own host work, the
                                caller's part (truncation, module-array stock) outside
                                the entry calls                                       */
} nrg_stats;
NRG_API int nrg_context_get_stats(const nrg_context* ctx, nrg_stats* out);
NRG_API int nrg_context_reset_stats(nrg_context* ctx);
NRG_API int nrg_context_set_profiling(nrg_context* ctx, int on);
/* Frees the device and pinned host storage a context keeps between runs (eigenvector
 * store, invariant matrices, workspaces); the model stays set and the next run
 * allocates again.  (No reference counterpart: the reference deallocates its module
 * arrays when the program ends.) */
NRG_API int nrg_context_release_storage(nrg_context* ctx);
NRG_API const char* nrg_last_error(void);
NRG_API const char* nrg_status_string(int status);
NRG_API int nrg_version(void);

/* ---- prepareBasis(iteration)  (prepareBasis.F90:1-119) --------------------------------
 * The product basis of the kept states of the last iteration with the states the new
 * site adds: basis(i*nOps + j) = (basis_output(i)%basis - operation(j, 1:nVar), reference
 * i, variation of i, operation j) (:42-57), sorted by sortBasisArray (module.F90:531-602:
 * by quantum numbers, then reference, with that exchange sort's order among equal keys),
 * then the sector table subspaceInfo = (basis, dimension, count_eigenvector, start_input)
 * (:63-114).  Integer bookkeeping on the host, as in the reference; it needs no context
 * and no device (the device-resident sweep calls the same code where it builds the
 * records on the host).  operation is the
 * Fortran (nOps, nVar+nChain) table; basis_input receives nb_old*nOps records;
 * numberOfSubspace receives the sector count, also when subspaceCapacity is too small
 * (NRG_ERR_INVALID). */
NRG_API int nrg_prepare_basis(int32_t numberOfVariation, int32_t numberOfOperation, int32_t numberOfChain,
                              const int32_t* operation, int32_t numberOfBasis_old, const int32_t* basis_output,
                              int32_t* basis_input, int32_t* subspaceInfo, int32_t subspaceCapacity,
                              int32_t* numberOfSubspace);

/* ---- truncation and reorder of postprocess(iteration)  (postprocess.F90:69-168) --------
 * eigenvalue (sector order, as diagonalization leaves it) is sorted stably
 * (sortWithIndex, :75); unless iteration is the first or the last or nb <= truncation,
 * the kept count is N_keep extended over energies within 1e-6 of E(N_keep) and then cut
 * back by 0.001 steps until it is at most 1.2 N_keep (:79-126); the kept states are put
 * back in index order (sortByIndex, :140) and followed by the discarded ones in energy
 * order, and eigenvalue and basis_output (may be NULL) are permuted in place (:143-160).
 * startTrancation and flag_truncation are hami's fields, updated at the first truncated
 * iteration (:83-86).  Host work: no context, no device. */
NRG_API int nrg_truncate(int32_t iteration, int32_t indexOfFirstIteration, int32_t numberOfIteration,
                         int32_t truncation, int32_t numberOfVariation, int32_t numberOfBasis, double* eigenvalue,
                         int32_t* basis_output, int32_t* numberOfBasis_kept, int32_t* startTrancation,
                         int32_t* flag_truncation);

/* ---- diagonalization(iteration, ismysubspace)  (diagonalization.F90:1-410) ----------
 * Replaces the routine called from nrgIteration.F90:23.  Per symmetry sector: assemble
 * the block Hamiltonian (diagonalization.F90:162-262), diagonalise it (dsyev 'V','U',
 * :267), chop |V| < 1e-14 (:273-280); then shift the eigenvalues by their minimum and
 * zero those <= 1e-12 (:353-356) and rebuild basis_output (:394-407).  ismysubspace of
 * the reference is not needed: one device owns all sectors. */
typedef struct nrg_diagonalization_io {
    int32_t numberOfSubspace;          /* in                                             */
    const int32_t* subspaceInfo;       /* in  [nsub*(nVar+3)]                            */
    int32_t numberOfBasis;             /* in  nb = numberOfBasis_old * nOps              */
    const int32_t* basis_input;        /* in  [nb*(nVar+3)]                              */
    int32_t numberOfBasis_old;         /* in                                             */
    const double* eigenvalue_old;      /* in  [nb_old]  eigenvalue of the last iteration */
    const double* invariant_matrix;    /* in  (nb_old, nb_old, nCM)                      */
    double* eigenvalue;                /* out [nb]                                       */
    double* eigenvector;               /* out [sizeOfEigenvector] column-major blocks    */
    int64_t sizeOfEigenvector;         /* in  capacity = sum over sectors of dimension^2 */
    int32_t* basis_output;             /* out [nb*(nVar+3)]                              */
    double* groundStateEnergy;         /* out eigenvalue(1) before the shift (:351)      */
} nrg_diagonalization_io;
NRG_API int nrg_diagonalization(nrg_context* ctx, int32_t iteration, const nrg_diagonalization_io* io);

/* ---- invariantMatrixDGEMM(iteration) and invariantMatrixForSpectrumDGEMM(iteration) ---
 * (invariantMatrixDGEMM.F90:1-394, invariantMatrixForSpectrumDGEMM.F90:1-392), called
 * from postprocess.F90:194,197 after truncation.  basis_output holds the kept states
 * first (numberOfBasis of them, postprocess.F90:143-160). */
typedef struct nrg_invariant_matrix_io {
    int32_t numberOfSubspace;          /* in                                             */
    const int32_t* subspaceInfo;       /* in  [nsub*(nVar+3)]                            */
    int32_t numberOfBasisFull;         /* in  states before truncation                   */
    const int32_t* basis_input;        /* in  [nb_full*(nVar+3)]                         */
    int32_t numberOfBasis;             /* in  kept states                                */
    const int32_t* basis_output;       /* in  [>= nb*(nVar+3)], kept prefix used         */
    const double* eigenvector;         /* in  [sizeOfEigenvector]                        */
    int64_t sizeOfEigenvector;         /* in                                             */
    int32_t numberOfBasis_old;         /* in  (spectrum variant) rows of the old matrix  */
    const double* invariant_matrix_spectrum_old; /* in (nb_old, nb_old, nMat) (spectrum) */
    double* invariant_matrix;          /* out (nb, nb, nCM) or (nb, nb, nMat)            */
} nrg_invariant_matrix_io;
NRG_API int nrg_invariant_matrix_dgemm(nrg_context* ctx, int32_t iteration,
                               const nrg_invariant_matrix_io* io);
NRG_API int nrg_invariant_matrix_for_spectrum_dgemm(nrg_context* ctx, int32_t iteration,
                                            const nrg_invariant_matrix_io* io);

/* ---- reducedDensityMatrixCalculation()  (reducedDensityMatrixDGEMM.F90:2-377) --------
 * Backward recursion rho_N = A rho_{N+1} A^T for N = numberOfIteration-1 .. startTrancation,
 * called from main.F90:200 after initializeReducedDensity.  mapFullSubspaceInfo is
 * indexed from iteration -1 (element 0 is mapFullSubspaceInfo(-1)). */
typedef struct nrg_reduced_density_io {
    int32_t numberOfIteration;
    int32_t startTrancation;
    const int32_t* mapFullSubspaceInfo;   /* in  (-1:numberOfIteration)                  */
    int32_t elementNumFullSubspace;       /* in                                          */
    int32_t* fullSubspaceInfo;            /* inout [n*(nVar+6)], start_matrix filled     */
    const int32_t* fullBasisInput;        /* in  [numFullBasisInput*(nVar+3)]            */
    int64_t numFullBasisInput;
    const int32_t* fullBasisOutput;       /* in  [numFullBasisOutput*(nVar+3)]           */
    int64_t numFullBasisOutput;
    const double* fullEigenvector;        /* in                                          */
    int64_t numFullEigenvector;
    double* reducedDensityMatrix;         /* inout [sizeOfReducedDensity]                */
    int64_t sizeOfReducedDensity;
    int32_t* pointReducedDensity;         /* inout                                       */
    double* trace;                        /* out, optional [numberOfIteration - startTrancation] */
} nrg_reduced_density_io;
NRG_API int nrg_reduced_density_matrix(nrg_context* ctx, const nrg_reduced_density_io* io);

/* ---- spikeZeroTemperature(iteration) / spikeCFS(iteration, numberOfBasisFull) --------
 * (calculateSpectrumDGEMM.F90:1-215 and :217-646), called from cfsSpectrumCalculation
 * (module.F90:1700,1702) after getRestore.  Spikes are binned onto the logarithmic grid
 * of binningSpike (module.F90:1210-1254) and added to the weight column of the bins. */
typedef struct nrg_spike_io {
    int32_t numberOfSubspace;
    const int32_t* subspaceInfo;          /* [nsub*(nVar+3)] of this iteration           */
    int32_t numberOfBasis;                /* kept states (hami%numberOfBasis)            */
    int32_t numberOfBasisFull;            /* all states of this iteration                */
    const int32_t* basis_input;           /* [nb_full*(nVar+3)]                          */
    const int32_t* basis_output;          /* [nb_full*(nVar+3)]                          */
    const double* eigenvalue;             /* [nb_full]                                   */
    const double* eigenvector;            /* [sizeOfEigenvector]                         */
    int64_t sizeOfEigenvector;
    int32_t numberOfBasis_old;
    const double* invariant_matrix_spectrum; /* (nb_old, nb_old, nMat) of iteration-1   */
    const int32_t* fullSubspaceInfo;      /* spikeCFS only                               */
    const int32_t* mapFullSubspaceInfo;   /* spikeCFS only, from iteration -1            */
    int32_t elementNumFullSubspace;       /* spikeCFS only                               */
    const double* reducedDensityMatrix;   /* spikeCFS only                               */
    int64_t sizeOfReducedDensity;
    int32_t numberOfBin;
    double* binnedSpikePositive;          /* inout (numberOfBin*nMat, 2)                 */
    double* binnedSpikeNegative;          /* inout (numberOfBin*nMat, 2)                 */
    double* total_sum;                    /* out, optional [4*nMat]: raw negative, raw
                                             positive, binned negative, binned positive
                                             (spikeCFS check, :559-596)                  */
} nrg_spike_io;
NRG_API int nrg_spike_zero_temperature(nrg_context* ctx, int32_t iteration, const nrg_spike_io* io);
NRG_API int nrg_spike_cfs(nrg_context* ctx, int32_t iteration, const nrg_spike_io* io);

/* ---- one symmetric block without any device allocation --------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device memory: a
 * host application whose pool allocator owns the whole device, or a caller that must not
 * trigger the implicit device synchronisation of cudaMalloc/cudaFree inside a pipelined
 * stream of work.  Diagonalises one symmetric FP64 block (column-major, order n <=
 * NRG_NOALLOC_MAX_ORDER) with the same per-sector eigensolver kernel nrg_diagonalization
 * uses (without the |V| < 1e-14 chop): eigenvalues ascending, eigenvectors in the same
 * column order.  H, eigenvalues and eigenvectors are caller-owned device arrays (H may
 * equal eigenvectors).  No context is needed: the call runs on the current device and on
 * `stream` (NULL = default stream), and returns after the stream has drained.
 * Its workspace is a static device array of about 417 KB, created on a device when the
 * library's device code is loaded there (with lazy module loading, the CUDA default, at
 * the first call on that device: a warm-up call during the caller's set-up keeps that
 * load out of later work) and held until the process exits.  The first call on a device
 * looks up that array's address (cudaGetSymbolAddress) and keeps it for the device's
 * CUDA context; after a device reset the next call looks it up again.  So make the first
 * call before any stream capture.  Each call copies a small descriptor to the device,
 * reads a status word back and returns after `stream` has drained.  Every call shares the
 * one array, which keeps the previous call's contents (the call clears its status word
 * itself): calls that overlap on the GPU (concurrent streams, threads) race and must be
 * serialised by the caller.  H, eigenvalues and eigenvectors must be memory of the current
 * device or managed memory (NRG_ERR_INVALID otherwise).  A block holding NaN or Inf
 * returns NRG_ERR_NUMERIC.  Orders above the maximum return NRG_ERR_TOO_LARGE. */
#define NRG_NOALLOC_MAX_ORDER 128
NRG_API int nrg_block_eigh_noalloc(const double* H, int32_t n, double* eigenvalues,
                                   double* eigenvectors, void* stream);

/* ---- pinned host memory for module arrays ------------------------------------------
 * No counterpart in the reference (its module arrays are Fortran allocatables).  Page-
 * locked host memory for the arrays that cross the boundary on every iteration
 * (eigenvector, invariant_matrix, invariant_matrix_spectrum): copies between it and the
 * device run at full link speed without an extra staging copy.  Optional: every entry
 * point accepts arrays from any allocator.  A Fortran caller maps the block with
 * c_f_pointer.  nrg_host_free(NULL) is a no-op. */
NRG_API int nrg_host_alloc(size_t bytes, void** out);
NRG_API int nrg_host_free(void* p);

/* ---- whole run: main.F90:142-252 with everything device resident ---------------------
 * Replays the reference's driver (forward NRG sweep, backward reduced density matrices,
 * CFS spectrum at T = 0) on one device.  Initial state as read from initial.dat.  In the
 * device-resident run (host_drop_in = 0) the per-state bookkeeping between iterations
 * also runs on the device: the truncation of postprocess (postprocess.F90:69-140) and,
 * after the first iteration, the basis records and row lists of prepareBasis
 * (prepareBasis.F90:31-114); the host keeps a few integers per sector.  Models whose
 * operations change the quantum numbers alike (ties in sortBasisArray's exchange sort)
 * build the records on the host, where that exchange sequence is replayed.  Setting the
 * environment variable NRG_HOST_TABLES=1 keeps all the bookkeeping on the host;
 * NRG_CHECK_TABLES=1 compares the device's tables with the host's at every iteration and
 * fails the run (NRG_ERR_STATE) on any difference. */
typedef struct nrg_run_input {
    int32_t numberOfBasis;                /* impurity basis size                        */
    const int32_t* basis_output;          /* [nb*(nVar+3)]                              */
    const double* eigenvalue;             /* [nb]                                       */
    const double* invariant_matrix;       /* (nb, nb, nCM)                              */
    const double* invariant_matrix_spectrum; /* (nb, nb, nMat)                          */
    int32_t spectrum;                     /* 0: forward sweep only                     */
    int32_t host_drop_in;                 /* 1: every routine goes through the drop-in
                                             entry points with host arrays (the
                                             Fortran caller's data flow)               */
    double temperature;                   /* 0: the reference's T = 0 CFS spectrum;
                                             > 0 (device-resident run only): the
                                             full-density-matrix spectrum at this
                                             temperature (energy units of the band
                                             half-width D), no reference counterpart:
                                             Weichselbaum and von Delft, PRL 99,
                                             076402 (2007); rdmTrace then holds, per
                                             shell N, the kept-space trace plus the
                                             weight discarded up to N (1)              */
    /* restart.dat of the CFS phase (saveRestart / loadRestart, module.F90:1710-1890;
     * main.F90:165-224), in the reference's byte layout: Fortran stream output of the
     * restore stock, the full stock, the density matrices and the bins.  Drop-in replay
     * only (host_drop_in = 1) and with the spectrum on; NRG_ERR_INVALID otherwise, and
     * for a missing, broken or foreign file. */
    const char* restart_file;             /* path; NULL or "": "restart.dat"            */
    int32_t save_restart;                 /* param%saveRestart: rewrite the file before
                                             every CFS step (after the file's step when
                                             resuming)                                  */
    int32_t load_restart;                 /* param%loadRestart: skip the NRG sweep and the
                                             density matrices and resume the CFS loop at
                                             the file's iteration; kept and
                                             numberOfBasisFull come from the file, the
                                             sweep's other outputs are NaN             */
    int32_t host_arrays_pageable;         /* drop-in replay: 1 keeps the emulated caller's
                                             large module arrays (eigenvector, invariant
                                             matrices, the full stock) in pageable memory,
                                             as a Fortran allocatable is; 0 in page-locked
                                             memory                                      */
} nrg_run_input;

typedef struct nrg_run_output {
    int32_t numberOfBin;                  /* out                                        */
    double* binnedSpikePositive;          /* out, capacity numberOfBin*nMat*2 (may be NULL) */
    double* binnedSpikeNegative;          /* out                                        */
    int64_t binCapacity;                  /* in  doubles available in each bin array    */
    int32_t startTrancation;              /* out                                        */
    int32_t* kept;                        /* out, optional [nIter-first+1]              */
    int32_t* numberOfBasisFull;           /* out, optional [nIter-first+1]              */
    double* groundStateEnergy;            /* out, optional [nIter-first+1]              */
    double* rdmTrace;                     /* out, optional [nIter+1]: trace at N         */
    double* flow;                         /* out, optional [nIter-first+1]*flowStride:
                                             lowest kept energies per iteration         */
    int32_t flowStride;
    double* finalEigenvalue;              /* out, optional [finalCapacity]              */
    int32_t finalCapacity;
    double* phaseSeconds;                 /* out, optional [4]: nrg sweep, rdm, cfs, total
                                             (device events)                            */
    double* thermo;                       /* out, optional [nIter-first+1]*3: Cn, Sn, Xn of
                                             calcThermo (module.F90:1931-1982, called at
                                             postprocess.F90:62) per iteration, computed on
                                             the device in the device-resident run; NaN in
                                             the drop-in replay, whose caller computes
                                             them on the host as the reference does     */
} nrg_run_output;
NRG_API int nrg_run(nrg_context* ctx, const nrg_run_input* in, nrg_run_output* out);

/* ---- many independent impurity instances on one device ------------------------------
 * The reference runs one impurity per MPI job; loadbalance.F90:102-186
 * (loadbalanceDiagonalization2) spreads the sectors of one iteration over the ranks by a
 * greedy d^3 cost.  On one B200 a single instance leaves most SMs idle (its work is a
 * chain of latency-bound sector solves), so independent instances (parameter sweeps)
 * run side by side: count instances, each a context with its model set (distinct
 * contexts, all on one device), as nrg_run calls on up to `concurrency` host threads
 * (concurrency < 1: one per instance), each instance on its own CUDA stream (a context
 * whose stream is NULL gets a non-blocking stream for the call).  Instances start in
 * array order; callers sort them by estimated cost, largest first.  statuses[i]
 * (optional) receives each instance's status; the return value is the status of the
 * first failing instance (all instances run to the end), or NRG_OK. */
/* ---- log-Gaussian broadening of a binned spectrum -----------------------------------
 * No reference counterpart: the reference writes raw bins (binnedSpikePositive/Negative,
 * main.F90:204-252) and leaves the smoothing to post-processing.  The standard NRG kernel
 * (Bulla, Costi and Pruschke, Rev. Mod. Phys. 80, 395 (2008), Sec. V.A):
 *   A[m*nOmega + k] = sum_i w_i exp(-b^2/4) / (b |E_i| sqrt(pi)) exp(-(ln(omega_k/E_i)/b)^2)
 * over the bins i of matrix type m with omega_k E_i > 0.  bins is a binnedSpike array as
 * spikeCFS fills it, Fortran (numberOfBin*nMat, 2): energies, then weights; pass the
 * positive and the negative array in turn.  Host or device pointers. */
NRG_API int nrg_broaden_log_gaussian(nrg_context* ctx, const double* bins, int32_t numberOfBin, int32_t nMat,
                                     double b, const double* omega, int32_t nOmega, double* A);

#define NRG_BATCH_RELEASE 1   /* flags: release each context's storage when its instance ends,
                                 so that device memory holds only the instances in flight */
NRG_API int nrg_run_batch(nrg_context* const* ctxs, const nrg_run_input* in, nrg_run_output* out,
                          int32_t count, int32_t concurrency, int32_t flags, int32_t* statuses);

#ifdef __cplusplus
}
#endif
#endif /* NRG_B200_H */
