"""ctypes mirror of include/nrg_b200.h and a thin Python front end.

The product path is the CUDA library ``libnrgb200.so`` built next to this file.  Loading
fails loudly when it is missing; every compute call fails with ``NrgError`` when no CUDA
device is usable.  There is no CPU fallback.

The methods of :class:`Context` keep the reference's routine names and argument meaning
(module arrays of the Fortran code, 1-based integer records, column-major real arrays):

======================================  ==============================================
reference routine                        method
======================================  ==============================================
diagonalization (diagonalization.F90)    ``Context.diagonalization``
invariantMatrixDGEMM                     ``Context.invariant_matrix_dgemm``
invariantMatrixForSpectrumDGEMM          ``Context.invariant_matrix_for_spectrum_dgemm``
reducedDensityMatrixCalculation          ``Context.reduced_density_matrix``
spikeZeroTemperature                     ``Context.spike_zero_temperature``
spikeCFS                                 ``Context.spike_cfs``
main.F90 (whole run, device resident)    ``Context.run``
======================================  ==============================================
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_double, c_int32, c_int64, c_void_p
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libnrgb200.so")

NRG_OK = 0
STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "out of device memory",
          4: "block too large", 5: "no usable CUDA device", 6: "unsupported input",
          7: "call sequence error", 8: "numerical failure", 9: "device wait timed out"}

# every entry point declared in include/nrg_b200.h
EXPORTS = [
    "nrg_context_create", "nrg_context_destroy", "nrg_context_set_stream",
    "nrg_context_set_model", "nrg_context_launch_count", "nrg_last_error", "nrg_status_string",
    "nrg_version", "nrg_diagonalization", "nrg_invariant_matrix_dgemm",
    "nrg_invariant_matrix_for_spectrum_dgemm", "nrg_reduced_density_matrix",
    "nrg_spike_zero_temperature", "nrg_spike_cfs", "nrg_run", "nrg_context_get_stats",
    "nrg_context_reset_stats", "nrg_context_set_profiling", "nrg_block_eigh_noalloc",
    "nrg_host_alloc", "nrg_host_free", "nrg_run_batch", "nrg_context_release_storage",
    "nrg_broaden_log_gaussian", "nrg_prepare_basis", "nrg_truncate",
]


class NrgError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        super().__init__(f"{where}: {STATUS.get(status, status)} ({detail})")


_pi32 = POINTER(c_int32)
_pf64 = POINTER(c_double)


class NrgModel(ctypes.Structure):
    _fields_ = [
        ("numberOfIteration", c_int32), ("numberOfChain", c_int32), ("numberOfVariation", c_int32),
        ("conservationBlock", c_int32 * 4), ("numberOfMatrix", c_int32),
        ("numberOfConductionMatrix", c_int32), ("numberOfCoefficient", c_int32),
        ("numberOfOperation", c_int32), ("numberOfBCSCoefficient", c_int32),
        ("indexOfFirstIteration", c_int32), ("flag_spectrum", c_int32), ("flag_BCS", c_int32),
        ("bandWidth", c_double), ("ztrick", c_double), ("Lambda", c_double),
        ("scalingType", c_int32), ("truncation", c_int32),
        ("operation", _pi32), ("coefficient_invariant_matrix_type", _pi32),
        ("coefficient_invariant_matrix", _pf64), ("coefficient_diagonalization_type", _pi32),
        ("coefficient_diagonalization", _pf64), ("chain_diagonal", _pf64),
        ("chain_nondiagonal", _pf64), ("chain_BCS", _pf64), ("coefficient_BCS", _pi32),
        ("coefficient_invariant_matrix_spectrum", _pf64),
        ("conservation_difference_spectrum", _pi32), ("positiveSpectrumOperation", _pi32),
        ("negativeSpectrumOperation", _pi32),
    ]


class DiagIO(ctypes.Structure):
    _fields_ = [
        ("numberOfSubspace", c_int32), ("subspaceInfo", _pi32), ("numberOfBasis", c_int32),
        ("basis_input", _pi32), ("numberOfBasis_old", c_int32), ("eigenvalue_old", _pf64),
        ("invariant_matrix", _pf64), ("eigenvalue", _pf64), ("eigenvector", _pf64),
        ("sizeOfEigenvector", c_int64), ("basis_output", _pi32), ("groundStateEnergy", _pf64),
    ]


class InvMatIO(ctypes.Structure):
    _fields_ = [
        ("numberOfSubspace", c_int32), ("subspaceInfo", _pi32), ("numberOfBasisFull", c_int32),
        ("basis_input", _pi32), ("numberOfBasis", c_int32), ("basis_output", _pi32),
        ("eigenvector", _pf64), ("sizeOfEigenvector", c_int64), ("numberOfBasis_old", c_int32),
        ("invariant_matrix_spectrum_old", _pf64), ("invariant_matrix", _pf64),
    ]


class RdmIO(ctypes.Structure):
    _fields_ = [
        ("numberOfIteration", c_int32), ("startTrancation", c_int32),
        ("mapFullSubspaceInfo", _pi32), ("elementNumFullSubspace", c_int32),
        ("fullSubspaceInfo", _pi32), ("fullBasisInput", _pi32), ("numFullBasisInput", c_int64),
        ("fullBasisOutput", _pi32), ("numFullBasisOutput", c_int64),
        ("fullEigenvector", _pf64), ("numFullEigenvector", c_int64),
        ("reducedDensityMatrix", _pf64), ("sizeOfReducedDensity", c_int64),
        ("pointReducedDensity", _pi32), ("trace", _pf64),
    ]


class SpikeIO(ctypes.Structure):
    _fields_ = [
        ("numberOfSubspace", c_int32), ("subspaceInfo", _pi32), ("numberOfBasis", c_int32),
        ("numberOfBasisFull", c_int32), ("basis_input", _pi32), ("basis_output", _pi32),
        ("eigenvalue", _pf64), ("eigenvector", _pf64), ("sizeOfEigenvector", c_int64),
        ("numberOfBasis_old", c_int32), ("invariant_matrix_spectrum", _pf64),
        ("fullSubspaceInfo", _pi32), ("mapFullSubspaceInfo", _pi32),
        ("elementNumFullSubspace", c_int32), ("reducedDensityMatrix", _pf64),
        ("sizeOfReducedDensity", c_int64), ("numberOfBin", c_int32),
        ("binnedSpikePositive", _pf64), ("binnedSpikeNegative", _pf64), ("total_sum", _pf64),
    ]


class RunInput(ctypes.Structure):
    _fields_ = [
        ("numberOfBasis", c_int32), ("basis_output", _pi32), ("eigenvalue", _pf64),
        ("invariant_matrix", _pf64), ("invariant_matrix_spectrum", _pf64),
        ("spectrum", c_int32), ("host_drop_in", c_int32), ("temperature", c_double),
        ("restart_file", ctypes.c_char_p), ("save_restart", c_int32), ("load_restart", c_int32),
        ("host_arrays_pageable", c_int32),
    ]


class RunOutput(ctypes.Structure):
    _fields_ = [
        ("numberOfBin", c_int32), ("binnedSpikePositive", _pf64), ("binnedSpikeNegative", _pf64),
        ("binCapacity", c_int64), ("startTrancation", c_int32), ("kept", _pi32),
        ("numberOfBasisFull", _pi32), ("groundStateEnergy", _pf64), ("rdmTrace", _pf64),
        ("flow", _pf64), ("flowStride", c_int32), ("finalEigenvalue", _pf64),
        ("finalCapacity", c_int32), ("phaseSeconds", _pf64), ("thermo", _pf64),
    ]


class Stats(ctypes.Structure):
    _fields_ = [("launches", c_int64), ("syev_launches", c_int64), ("syev_ms", c_double),
                ("syev_flops", c_double), ("h2d_bytes", c_int64), ("d2h_bytes", c_int64),
                ("tri_launches", c_int64), ("tri_ms", c_double), ("tri_flops", c_double),
                ("tri_bytes", c_double), ("entry_in_s", c_double), ("entry_compute_s", c_double),
                ("entry_out_s", c_double), ("entry_calls", c_int64), ("replay_host_s", c_double)]


_lib = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load libnrgb200.so (raises OSError when it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise OSError(f"{path} is missing: build it with nrg-mpi_b200/build.py")
    lib = ctypes.CDLL(path)
    lib.nrg_context_create.argtypes = [POINTER(c_void_p), ctypes.c_int]
    lib.nrg_context_destroy.argtypes = [c_void_p]
    lib.nrg_context_set_stream.argtypes = [c_void_p, c_void_p]
    lib.nrg_context_set_model.argtypes = [c_void_p, POINTER(NrgModel)]
    lib.nrg_context_launch_count.argtypes = [c_void_p]
    lib.nrg_context_launch_count.restype = c_int64
    lib.nrg_last_error.restype = ctypes.c_char_p
    lib.nrg_status_string.restype = ctypes.c_char_p
    lib.nrg_status_string.argtypes = [ctypes.c_int]
    lib.nrg_diagonalization.argtypes = [c_void_p, c_int32, POINTER(DiagIO)]
    lib.nrg_invariant_matrix_dgemm.argtypes = [c_void_p, c_int32, POINTER(InvMatIO)]
    lib.nrg_invariant_matrix_for_spectrum_dgemm.argtypes = [c_void_p, c_int32, POINTER(InvMatIO)]
    lib.nrg_reduced_density_matrix.argtypes = [c_void_p, POINTER(RdmIO)]
    lib.nrg_spike_zero_temperature.argtypes = [c_void_p, c_int32, POINTER(SpikeIO)]
    lib.nrg_spike_cfs.argtypes = [c_void_p, c_int32, POINTER(SpikeIO)]
    lib.nrg_run.argtypes = [c_void_p, POINTER(RunInput), POINTER(RunOutput)]
    lib.nrg_run_batch.argtypes = [POINTER(c_void_p), POINTER(RunInput), POINTER(RunOutput), c_int32, c_int32,
                                  c_int32, POINTER(c_int32)]
    lib.nrg_context_release_storage.argtypes = [c_void_p]
    lib.nrg_broaden_log_gaussian.argtypes = [c_void_p, POINTER(c_double), c_int32, c_int32, c_double,
                                             POINTER(c_double), c_int32, POINTER(c_double)]
    lib.nrg_prepare_basis.argtypes = [c_int32, c_int32, c_int32, POINTER(c_int32), c_int32, POINTER(c_int32),
                                      POINTER(c_int32), POINTER(c_int32), c_int32, POINTER(c_int32)]
    lib.nrg_truncate.argtypes = [c_int32, c_int32, c_int32, c_int32, c_int32, c_int32, POINTER(c_double),
                                 POINTER(c_int32), POINTER(c_int32), POINTER(c_int32), POINTER(c_int32)]
    lib.nrg_context_get_stats.argtypes = [c_void_p, POINTER(Stats)]
    lib.nrg_context_reset_stats.argtypes = [c_void_p]
    lib.nrg_context_set_profiling.argtypes = [c_void_p, ctypes.c_int]
    _lib = lib
    return lib


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32).reshape(-1))


def _i32f(a) -> np.ndarray:
    """Fortran (column-major) flat int32 copy of a 2-D table."""
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32).ravel(order="F"))


def _f64f(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel(order="F"))


def _p(a, t):
    return None if a is None else a.ctypes.data_as(POINTER(t))


def prepare_basis(operation, nVar: int, basis_output):
    """nrg_prepare_basis (prepareBasis.F90:1-119): the product basis of the kept records
    ``basis_output`` (nb_old, nVar+3) with the new site's ``operation`` table (nOps,
    nVar+nChain); returns (basis_input (nb_old*nOps, nVar+3), subspaceInfo (nsub, nVar+3)),
    1-based values as in the reference.  Host integer work: no context, no device."""
    lib = load_library()
    op = np.asarray(operation, dtype=np.int32)
    nOps, ncol = op.shape
    rs = nVar + 3
    bo = np.ascontiguousarray(np.asarray(basis_output, dtype=np.int32).reshape(-1, rs))
    nb = bo.shape[0] * nOps
    bi = np.zeros((nb, rs), dtype=np.int32)
    cap = max(nb, 1)
    si = np.zeros((cap, rs), dtype=np.int32)
    opf = _i32f(op)
    nsub = c_int32(0)
    rc = lib.nrg_prepare_basis(nVar, nOps, ncol - nVar, _p(opf, c_int32), bo.shape[0], _p(bo, c_int32),
                               _p(bi, c_int32), _p(si, c_int32), cap, ctypes.byref(nsub))
    if rc != 0:
        raise NrgError(rc, "nrg_prepare_basis", lib.nrg_last_error().decode(errors="replace"))
    return bi, si[:nsub.value].copy()


def truncate(iteration: int, first: int, nIter: int, n_keep: int, nVar: int, eigenvalue, basis_output,
             startTrancation: int, flag_truncation: bool):
    """nrg_truncate (postprocess.F90:69-168): returns (eigenvalue, basis_output) reordered
    (kept states in index order, then the discarded ones in energy order), the kept count
    and the updated (startTrancation, flag_truncation).  Host work: no context, no device."""
    lib = load_library()
    E = np.array(eigenvalue, dtype=np.float64, copy=True)
    bo = np.ascontiguousarray(np.array(basis_output, dtype=np.int32, copy=True).reshape(len(E), nVar + 3))
    kept, s_t, f_t = c_int32(0), c_int32(int(startTrancation)), c_int32(int(bool(flag_truncation)))
    rc = lib.nrg_truncate(iteration, first, nIter, n_keep, nVar, len(E), _p(E, c_double), _p(bo, c_int32),
                          ctypes.byref(kept), ctypes.byref(s_t), ctypes.byref(f_t))
    if rc != 0:
        raise NrgError(rc, "nrg_truncate", lib.nrg_last_error().decode(errors="replace"))
    return E, bo, kept.value, s_t.value, bool(f_t.value)


class Context:
    """One CUDA device with the model tables of one NRG problem."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        self._h = c_void_p()
        self._check(self.lib.nrg_context_create(ctypes.byref(self._h), device), "nrg_context_create")
        self._keep = []
        self.inp = None

    def _check(self, rc: int, where: str):
        if rc != NRG_OK:
            raise NrgError(rc, where, self.lib.nrg_last_error().decode(errors="replace"))

    def close(self):
        if self._h:
            self.lib.nrg_context_destroy(self._h)
            self._h = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def launch_count(self) -> int:
        return int(self.lib.nrg_context_launch_count(self._h))

    def set_stream(self, stream_handle: int):
        self._check(self.lib.nrg_context_set_stream(self._h, c_void_p(stream_handle)), "set_stream")

    def broaden_log_gaussian(self, bins, numberOfBin: int, nMat: int, b: float, omega):
        """nrg_broaden_log_gaussian: A of shape (nMat, len(omega)) from one binnedSpike array."""
        bins = np.asfortranarray(bins, dtype=np.float64)
        if bins.shape != (numberOfBin * nMat, 2):
            raise NrgError(1, "broaden_log_gaussian", f"bins shape {bins.shape}")
        om = np.ascontiguousarray(omega, dtype=np.float64)
        A = np.zeros(nMat * om.size)
        self._check(self.lib.nrg_broaden_log_gaussian(self._h, _p(bins, c_double), numberOfBin, nMat, float(b),
                                                      _p(om, c_double), om.size, _p(A, c_double)),
                    "broaden_log_gaussian")
        return A.reshape(nMat, om.size)

    def release_storage(self):
        """Frees the device storage kept between runs (the model stays set)."""
        self._check(self.lib.nrg_context_release_storage(self._h), "release_storage")

    def set_profiling(self, on: bool = True):
        self._check(self.lib.nrg_context_set_profiling(self._h, int(bool(on))), "set_profiling")

    def reset_stats(self):
        self._check(self.lib.nrg_context_reset_stats(self._h), "reset_stats")

    def stats(self) -> dict:
        s = Stats()
        self._check(self.lib.nrg_context_get_stats(self._h, ctypes.byref(s)), "get_stats")
        return {k: getattr(s, k) for k, _ in Stats._fields_}

    # ------------------------------------------------------------------
    def set_model(self, inp):
        """setupHamiltonian + read_initial_basis: ``inp`` is a ``model.NrgInput``."""
        cd, cn, cb = inp.rescaled_chains()
        arrs = dict(
            operation=_i32f(inp.operation),
            cim_t=_i32f(inp.coefficient_invariant_matrix_type),
            cim=_f64f(inp.coefficient_invariant_matrix),
            cd_t=_i32f(inp.coefficient_diagonalization_type),
            cdd=_f64f(inp.coefficient_diagonalization),
            chd=_f64f(cd), chn=_f64f(cn),
            chb=None if cb is None else _f64f(cb),
            cbcs=None if inp.coefficient_BCS is None else _i32f(inp.coefficient_BCS),
        )
        if inp.flag_spectrum:
            arrs.update(cspec=_f64f(inp.coefficient_invariant_matrix_spectrum),
                        cds=_i32f(inp.conservation_difference_spectrum),
                        pos=_i32f(inp.positiveSpectrumOperation),
                        neg=_i32f(inp.negativeSpectrumOperation))
        m = NrgModel()
        m.numberOfIteration = inp.numberOfIteration
        m.numberOfChain = inp.numberOfChain
        m.numberOfVariation = inp.numberOfVariation
        cbk = np.asarray(inp.conservationBlock, dtype=np.int32)
        m.conservationBlock[:] = [int(cbk[0, 0]), int(cbk[1, 0]), int(cbk[0, 1]), int(cbk[1, 1])]
        m.numberOfMatrix = inp.numberOfMatrix if inp.flag_spectrum else 0
        m.numberOfConductionMatrix = inp.numberOfConductionMatrix
        m.numberOfCoefficient = inp.numberOfCoefficient
        m.numberOfOperation = inp.numberOfOperation
        m.numberOfBCSCoefficient = inp.numberOfBCSCoefficient
        m.indexOfFirstIteration = inp.indexOfFirstIteration
        m.flag_spectrum = int(bool(inp.flag_spectrum))
        m.flag_BCS = int(bool(inp.flag_BCS))
        m.bandWidth, m.ztrick, m.Lambda = inp.bandWidth, inp.ztrick, inp.Lambda
        m.scalingType, m.truncation = inp.scalingType, inp.truncation
        m.operation = _p(arrs["operation"], c_int32)
        m.coefficient_invariant_matrix_type = _p(arrs["cim_t"], c_int32)
        m.coefficient_invariant_matrix = _p(arrs["cim"], c_double)
        m.coefficient_diagonalization_type = _p(arrs["cd_t"], c_int32)
        m.coefficient_diagonalization = _p(arrs["cdd"], c_double)
        m.chain_diagonal = _p(arrs["chd"], c_double)
        m.chain_nondiagonal = _p(arrs["chn"], c_double)
        m.chain_BCS = _p(arrs["chb"], c_double)
        m.coefficient_BCS = _p(arrs["cbcs"], c_int32)
        if inp.flag_spectrum:
            m.coefficient_invariant_matrix_spectrum = _p(arrs["cspec"], c_double)
            m.conservation_difference_spectrum = _p(arrs["cds"], c_int32)
            m.positiveSpectrumOperation = _p(arrs["pos"], c_int32)
            m.negativeSpectrumOperation = _p(arrs["neg"], c_int32)
        self._check(self.lib.nrg_context_set_model(self._h, ctypes.byref(m)), "set_model")
        self.inp = inp
        return self

    # ------------------------------------------------------------------
    def diagonalization(self, iteration: int, subspaceInfo, basis_input, eigenvalue_old,
                        invariant_matrix):
        """diagonalization(iteration, ismysubspace) with the module arrays as arguments."""
        si = _i32(subspaceInfo)
        bi = _i32(basis_input)
        nVar = self.inp.numberOfVariation
        rs = nVar + 3
        nsub, nb = si.size // rs, bi.size // rs
        dims = si.reshape(nsub, rs)[:, nVar].astype(np.int64)
        size = int(np.sum(dims * dims))
        # numberOfBasis_old is the order of the old invariant matrix; eigenvalue may hold
        # more entries (the discarded states follow the kept ones, postprocess.F90:143-160)
        im_arr = np.asarray(invariant_matrix, dtype=np.float64)
        nbo = int(im_arr.shape[0])
        if im_arr.shape != (nbo, nbo, self.inp.numberOfConductionMatrix):
            raise ValueError(f"invariant_matrix must be (nb_old, nb_old, nCM), got {im_arr.shape}")
        eo = np.ascontiguousarray(np.asarray(eigenvalue_old, dtype=np.float64).reshape(-1)[:nbo])
        if eo.size != nbo:
            raise ValueError("eigenvalue_old shorter than numberOfBasis_old")
        im = _f64f(im_arr)
        E = np.zeros(nb)
        V = np.zeros(size)
        bo = np.zeros(nb * rs, dtype=np.int32)
        gs = c_double(0.0)
        io = DiagIO(nsub, _p(si, c_int32), nb, _p(bi, c_int32), nbo, _p(eo, c_double),
                    _p(im, c_double), _p(E, c_double), _p(V, c_double), size, _p(bo, c_int32),
                    ctypes.pointer(gs))
        self._check(self.lib.nrg_diagonalization(self._h, iteration, ctypes.byref(io)),
                    "nrg_diagonalization")
        return E, V, bo.reshape(nb, rs), gs.value

    def _invmat(self, fn, iteration, subspaceInfo, basis_input, nb_kept, basis_output,
                eigenvector, ims_old=None, spec=False):
        si = _i32(subspaceInfo)
        bi = _i32(basis_input)
        bo = _i32(basis_output)
        rs = self.inp.numberOfVariation + 3
        V = np.ascontiguousarray(eigenvector, dtype=np.float64)
        nmat = self.inp.numberOfMatrix if spec else self.inp.numberOfConductionMatrix
        out = np.zeros(nb_kept * nb_kept * nmat)
        ims = None if ims_old is None else _f64f(ims_old)
        nbo = 0 if ims_old is None else int(np.asarray(ims_old).shape[0])
        io = InvMatIO(si.size // rs, _p(si, c_int32), bi.size // rs, _p(bi, c_int32), nb_kept,
                      _p(bo, c_int32), _p(V, c_double), V.size, nbo, _p(ims, c_double),
                      _p(out, c_double))
        self._check(fn(self._h, iteration, ctypes.byref(io)), fn.__name__)
        return out.reshape((nb_kept, nb_kept, nmat), order="F")

    def invariant_matrix_dgemm(self, iteration, subspaceInfo, basis_input, nb_kept, basis_output,
                               eigenvector):
        return self._invmat(self.lib.nrg_invariant_matrix_dgemm, iteration, subspaceInfo,
                            basis_input, nb_kept, basis_output, eigenvector)

    def invariant_matrix_for_spectrum_dgemm(self, iteration, subspaceInfo, basis_input, nb_kept,
                                            basis_output, eigenvector, ims_old):
        return self._invmat(self.lib.nrg_invariant_matrix_for_spectrum_dgemm, iteration,
                            subspaceInfo, basis_input, nb_kept, basis_output, eigenvector,
                            ims_old=ims_old, spec=True)

    def reduced_density_matrix(self, numberOfIteration, startTrancation, mapFullSubspaceInfo,
                               fullSubspaceInfo, fullBasisInput, fullBasisOutput,
                               fullEigenvector, reducedDensityMatrix, pointReducedDensity):
        """reducedDensityMatrixCalculation(); returns (rdm, fullSubspaceInfo, point, trace)."""
        rs = self.inp.numberOfVariation + 3
        mp = _i32(mapFullSubspaceInfo)
        fsi = _i32(fullSubspaceInfo).copy()
        fbi = _i32(fullBasisInput)
        fbo = _i32(fullBasisOutput)
        fv = np.ascontiguousarray(fullEigenvector, dtype=np.float64)
        rdm = np.ascontiguousarray(reducedDensityMatrix, dtype=np.float64).copy()
        point = c_int32(int(pointReducedDensity))
        ntr = max(numberOfIteration - startTrancation, 1)
        trace = np.zeros(ntr)
        io = RdmIO(numberOfIteration, startTrancation, _p(mp, c_int32),
                   fsi.size // (self.inp.numberOfVariation + 6), _p(fsi, c_int32),
                   _p(fbi, c_int32), fbi.size // rs, _p(fbo, c_int32), fbo.size // rs,
                   _p(fv, c_double), fv.size, _p(rdm, c_double), rdm.size, ctypes.pointer(point),
                   _p(trace, c_double))
        self._check(self.lib.nrg_reduced_density_matrix(self._h, ctypes.byref(io)),
                    "nrg_reduced_density_matrix")
        return rdm, fsi.reshape(-1, self.inp.numberOfVariation + 6), point.value, trace

    def _spike(self, fn, iteration, R, binPos, binNeg, ims_prev, nb_old, full=None):
        rs = self.inp.numberOfVariation + 3
        si = _i32(R["subspaceInfo"])
        bi = _i32(R["basis_input"])
        bo = _i32(R["basis_output"])
        E = np.ascontiguousarray(R["eigenvalue"], dtype=np.float64)
        V = np.ascontiguousarray(R["eigenvector"], dtype=np.float64)
        if np.asarray(ims_prev).shape != (nb_old, nb_old, self.inp.numberOfMatrix):
            raise ValueError("invariant_matrix_spectrum must be (nb_old, nb_old, nMat)")
        ims = _f64f(ims_prev)
        tot = np.zeros(4 * self.inp.numberOfMatrix)
        nbin = binPos.shape[0] // self.inp.numberOfMatrix
        io = SpikeIO()
        io.numberOfSubspace = si.size // rs
        io.subspaceInfo = _p(si, c_int32)
        io.numberOfBasis = int(R["numberOfBasis"])
        io.numberOfBasisFull = bi.size // rs
        io.basis_input = _p(bi, c_int32)
        io.basis_output = _p(bo, c_int32)
        io.eigenvalue = _p(E, c_double)
        io.eigenvector = _p(V, c_double)
        io.sizeOfEigenvector = V.size
        io.numberOfBasis_old = nb_old
        io.invariant_matrix_spectrum = _p(ims, c_double)
        keep = []
        if full is not None:
            fsi, mp, rdm = (_i32(full["fullSubspaceInfo"]), _i32(full["map"]),
                            np.ascontiguousarray(full["rdm"], dtype=np.float64))
            keep += [fsi, mp, rdm]
            io.fullSubspaceInfo = _p(fsi, c_int32)
            io.mapFullSubspaceInfo = _p(mp, c_int32)
            io.elementNumFullSubspace = fsi.size // (self.inp.numberOfVariation + 6)
            io.reducedDensityMatrix = _p(rdm, c_double)
            io.sizeOfReducedDensity = rdm.size
        io.numberOfBin = nbin
        bp = np.asfortranarray(binPos)
        bn = np.asfortranarray(binNeg)
        io.binnedSpikePositive = bp.ctypes.data_as(POINTER(c_double))
        io.binnedSpikeNegative = bn.ctypes.data_as(POINTER(c_double))
        io.total_sum = _p(tot, c_double)
        self._check(fn(self._h, iteration, ctypes.byref(io)), fn.__name__)
        return bp, bn, tot.reshape(-1, 4)

    def spike_zero_temperature(self, iteration, R, binPos, binNeg, ims_prev, nb_old):
        return self._spike(self.lib.nrg_spike_zero_temperature, iteration, R, binPos, binNeg,
                           ims_prev, nb_old)

    def spike_cfs(self, iteration, R, binPos, binNeg, ims_prev, nb_old, full):
        return self._spike(self.lib.nrg_spike_cfs, iteration, R, binPos, binNeg, ims_prev,
                           nb_old, full=full)

    # ------------------------------------------------------------------
    def run(self, spectrum: bool = True, flow_stride: int = 8, final_capacity: int = 0,
            host_drop_in: bool = False, temperature: float = 0.0, restart_file: Optional[str] = None,
            save_restart: bool = False, load_restart: bool = False, host_pageable: bool = False):
        """main.F90:142-252; returns bins and per-iteration statistics.

        ``host_drop_in=True`` drives every routine through its drop-in entry point with
        host arrays (the Fortran caller's data flow) instead of keeping state on the device.
        ``temperature > 0`` (device-resident run) gives the full-density-matrix spectrum
        at that temperature instead of the reference's T = 0 CFS spectrum.
        ``save_restart`` / ``load_restart`` (drop-in replay with the spectrum on) are the
        reference's param%saveRestart / param%loadRestart: the file (``restart_file``,
        default "restart.dat") is rewritten before every CFS step, or the run resumes the
        CFS loop from it (module.F90:1710-1890, main.F90:165-224).
        ``host_pageable=True`` (drop-in replay) keeps the emulated caller's large module
        arrays in pageable memory, as a Fortran allocatable is, instead of page-locked memory.
        """
        args = self._run_args(spectrum, flow_stride, final_capacity, host_drop_in, temperature,
                              restart_file, save_restart, load_restart, host_pageable)
        self._check(self.lib.nrg_run(self._h, ctypes.byref(args["ri"]), ctypes.byref(args["ro"])), "nrg_run")
        return self._run_result(args)

    def _run_args(self, spectrum, flow_stride, final_capacity, host_drop_in, temperature=0.0,
                  restart_file=None, save_restart=False, load_restart=False, host_pageable=False):
        """Input and output records of nrg_run for this context (arrays kept alive here)."""
        inp = self.inp
        nb = inp.numberOfBasis
        a = dict(bo=_i32(inp.basis_output), E=np.ascontiguousarray(inp.eigenvalue, dtype=np.float64),
                 im=_f64f(inp.invariant_matrix),
                 ims=_f64f(inp.invariant_matrix_spectrum) if inp.flag_spectrum else None,
                 path=os.fsencode(restart_file) if restart_file else None)
        a["ri"] = RunInput(nb, _p(a["bo"], c_int32), _p(a["E"], c_double), _p(a["im"], c_double),
                           _p(a["ims"], c_double), int(bool(spectrum)), int(bool(host_drop_in)),
                           float(temperature), a["path"], int(bool(save_restart)), int(bool(load_restart)),
                           int(bool(host_pageable)))
        nit = inp.numberOfIteration - inp.indexOfFirstIteration + 1
        nmat = max(inp.numberOfMatrix, 1)
        nbin_cap = 20001
        a.update(bp=np.zeros(2 * nbin_cap * nmat), bn=np.zeros(2 * nbin_cap * nmat),
                 kept=np.zeros(nit, dtype=np.int32), nfull=np.zeros(nit, dtype=np.int32),
                 gse=np.zeros(nit), tr=np.full(inp.numberOfIteration + 1, np.nan),
                 flow=np.full(nit * flow_stride, np.nan), fin=np.zeros(max(final_capacity, 1)),
                 ph=np.zeros(4), thermo=np.full(3 * nit, np.nan), nit=nit, nmat=nmat,
                 spectrum=spectrum, flow_stride=flow_stride,
                 final_capacity=final_capacity)
        a["ro"] = RunOutput(0, _p(a["bp"], c_double), _p(a["bn"], c_double), a["bp"].size, 0,
                            _p(a["kept"], c_int32), _p(a["nfull"], c_int32), _p(a["gse"], c_double),
                            _p(a["tr"], c_double), _p(a["flow"], c_double), flow_stride,
                            _p(a["fin"], c_double), final_capacity, _p(a["ph"], c_double),
                            _p(a["thermo"], c_double))
        return a

    def _run_result(self, a):
        ro, nmat = a["ro"], a["nmat"]
        nbin = ro.numberOfBin
        if a["spectrum"] and self.inp.flag_spectrum and 2 * nbin * nmat > a["bp"].size:
            raise NrgError(4, "nrg_run", f"bin buffers too small for {nbin} bins")
        nw = nbin * nmat
        bp, bn = a["bp"], a["bn"]
        binPos = np.stack([bp[:nw], bp[nw:2 * nw]], axis=1)
        binNeg = np.stack([bn[:nw], bn[nw:2 * nw]], axis=1)
        return dict(numberOfBin=nbin, binPos=binPos, binNeg=binNeg, kept=a["kept"],
                    numberOfBasisFull=a["nfull"], groundStateEnergy=a["gse"], rdmTrace=a["tr"],
                    flow=a["flow"].reshape(a["nit"], a["flow_stride"]), startTrancation=ro.startTrancation,
                    finalEigenvalue=a["fin"][:a["final_capacity"]], phaseSeconds=a["ph"],
                    thermo=a["thermo"].reshape(a["nit"], 3))


def run_batch(contexts, spectrum: bool = True, concurrency: int = 0, flow_stride: int = 8,
              release: bool = False, temperature: float = 0.0):
    """nrg_run_batch: independent instances (distinct contexts on one device) side by side.
    ``release=True`` frees each context's run storage when its instance ends.
    ``temperature > 0`` gives every instance the full-density-matrix spectrum at that
    temperature (as ``Context.run``) instead of the T = 0 CFS spectrum.

    Returns (results, statuses): one result dict per context and the per-instance
    statuses; raises NrgError when any instance failed (every instance still ran).
    """
    if not contexts:
        return [], []
    lib = contexts[0].lib
    args = [c._run_args(spectrum, flow_stride, 0, False, temperature) for c in contexts]
    n = len(contexts)
    hs = (c_void_p * n)(*[c._h for c in contexts])
    ris = (RunInput * n)(*[a["ri"] for a in args])
    ros = (RunOutput * n)(*[a["ro"] for a in args])
    st = np.zeros(n, dtype=np.int32)
    rc = lib.nrg_run_batch(hs, ris, ros, n, int(concurrency), 1 if release else 0, _p(st, c_int32))
    if rc != 0:
        raise NrgError(rc, "nrg_run_batch", lib.nrg_last_error().decode(errors="replace"))
    results = []
    for i, (c, a) in enumerate(zip(contexts, args)):
        a["ro"] = ros[i]
        results.append(c._run_result(a))
    return results, st.tolist()
