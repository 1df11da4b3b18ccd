"""CPU oracle for the NRG hot path of eminamitani/nrg-mpi.

TEST INFRASTRUCTURE.  Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py`` may import this module, and only as the reference that results are
compared with or as the timed CPU baseline: the product never routes work through it.

What it is: a restatement, in numpy/scipy plus a small C helper, of the reference's
per-iteration NRG algorithm and of the CFS spectrum that follows it, with the reference's
index conventions (1-based values inside the integer records, Fortran column-major
matrices) and its quirks.  Each function cites the reference file:line it follows.

Third-party arithmetic at the boundary: the reference calls LAPACK ``dsyev('V','U')`` and
BLAS ``dgemm`` from MKL (Makefile:11, version not pinned by the reference).  The oracle
calls the same LAPACK driver (``dsyev`` with the upper triangle) through scipy's bundled
OpenBLAS/LAPACK and numpy's BLAS for the products.

PARITY UNPINNED against the reference binary: the reference ships no tests, inputs,
outputs or golden vectors, and it cannot be compiled here (no Fortran compiler, no MPI,
no MKL).  The oracle is pinned instead by (1) an exact known-answer case (the
non-interacting impurity, whose many-body NRG spectrum must reproduce the single-particle
eigenvalues and weights of the finite chain), (2) the loop-form legacy routines of the
reference (invariantMatrix.F90, invariantMatrixForSpectrum.F90, reducedDensityMatrix.F90,
calculateSpectrum.F90/spectrumElement) restated element by element in
``oracle/legacy_loops.py``, and (3) identities: RDM trace, orthonormality, spectral sum
rule.

Reference quirks restated on purpose (they affect parity):
* sortBasisArray is an unstable exchange sort (module.F90:531-602) -> C helper;
* groundStateEnergy is eigenvalue(1), the first element, not the minimum
  (diagonalization.F90:351);
* coefficient lookups: the last matching row wins (diagonalization.F90:195-213,
  invariantMatrixDGEMM.F90:248-254); in diagonalization the reference swap, once made
  by any matching row, persists;
* the eigenvector slice upper bound typo (invariantMatrixDGEMM.F90:223,227,
  invariantMatrixForSpectrumDGEMM.F90:224,228, module.F90:1063,1067) is read with
  column semantics (column isubl), as the legacy loops confirm;
* spikeZeroTemperature always uses column 1 of the ground-state sector
  (calculateSpectrumDGEMM.F90:107-111);
* no truncation at the first or the last iteration (postprocess.F90:79-81);
* betabar is the default-real literal 0.8 widened to double (module.F90:652);
* binningSpike edge handling with int() truncation and clamping (module.F90:1226-1251).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from typing import Dict, List, Optional, Tuple

import numpy as np
import scipy.linalg

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

NUMERICAL_THRESHOLD = 1.0e-12      # module.F90:5
EIGENVECTOR_THRESHOLD = 1.0e-14    # module.F90:6
DEGENERACY_THRESHOLD = 1.0e-8      # module.F90:7
TRUNCATION_THRESHOLD = 0.000001    # module.F90:629
TRUNCATION_LIMIT_SCALE = 1.2       # module.F90:630
MESH_OF_BIN = 1000                 # module.F90:964
LOG10_EMIN = -15.0                 # module.F90:970
BETABAR = float(np.float32(0.8))   # module.F90:652 (default-real literal)


# ------------------------------------------------------------------------------------
# C helper
# ------------------------------------------------------------------------------------
def build_helper() -> str:
    """Compile oracle/csrc/exchange_sort.c into oracle/_build/liboracle.so."""
    out_dir = os.path.join(_HERE, "_build")
    os.makedirs(out_dir, exist_ok=True)
    so = os.path.join(out_dir, "liboracle.so")
    src = os.path.join(_HERE, "csrc", "exchange_sort.c")
    if not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-O2", "-fPIC", "-shared", "-o", so, src])
    return so


def _lib():
    global _LIB
    if _LIB is None:
        _LIB = ctypes.CDLL(build_helper())
        _LIB.oracle_exchange_sort.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int]
        _LIB.oracle_exchange_sort.restype = None
    return _LIB


def exchange_sort(rec: np.ndarray, nvar: int) -> np.ndarray:
    """sortBasisArray (module.F90:531-602), in place on an (n, nvar+3) int32 array."""
    assert rec.dtype == np.int32 and rec.flags.c_contiguous
    _lib().oracle_exchange_sort(rec.ctypes.data, rec.shape[0], nvar)
    return rec


# ------------------------------------------------------------------------------------
# inputs (read_initial_basis.F90, module.F90:656-688, 846-880)
# ------------------------------------------------------------------------------------
def _namelist(path):
    txt = open(path).read()
    body = txt[txt.index("&"):]
    body = body[body.index("\n"):].rsplit("/", 1)[0]
    out, key = {}, None
    for tok in body.replace("\n", " ").split(","):
        tok = tok.strip()
        if not tok:
            continue
        if "=" in tok:
            k, v = tok.split("=", 1)
            key = k.strip()
            out[key] = [v.strip()]
        else:
            out[key].append(tok)
    return out


def _f(s):
    return float(s.lower().replace("d", "e"))


def _b(s):
    return s.strip().lower().strip(".").startswith("t")


class State:
    """The reference's module globals (module.F90 modules system, hamiltonian, spectrum)."""

    def __init__(self, directory: str):
        p = _namelist(os.path.join(directory, "parameter.txt"))
        h = _namelist(os.path.join(directory, "hamiltonianInfo.dat"))
        self.bandWidth = _f(p["bandWidth"][0])
        self.ztrick = _f(p["ztrick"][0])
        self.Lambda = _f(p["Lambda"][0])
        self.scalingType = int(p["scalingType"][0])
        self.truncation = int(p["truncation"][0])
        self.nIter = int(h["numberOfIteration"][0])
        self.nChain = int(h["numberOfChain"][0])
        self.nVar = int(h["numberOfVariation"][0])
        cb = [int(x) for x in h["conservationBlock"]]
        self.cb = np.array([[cb[0], cb[2]], [cb[1], cb[3]]])
        self.nMat = int(h["numberOfMatrix"][0])
        self.nCM = int(h["numberOfConductionMatrix"][0])
        self.nb = int(h["numberOfBasis"][0])
        self.nCoef = int(h["numberOfCoefficient"][0])
        self.nOps = int(h["numberOfOperation"][0])
        self.first = int(h["indexOfFirstIteration"][0])
        self.flag_spectrum = _b(h.get("flag_spectrum", [".false."])[0])
        self.flag_BCS = _b(h.get("flag_BCS", [".false."])[0])
        self.nBCS = int(h.get("numberOfBCSCoefficient", ["0"])[0])
        self.startTrancation = self.nIter + 1      # module.F90:879
        self.flag_truncation = False
        self._read_initial(os.path.join(directory, "initial.dat"))
        # main.F90:142-157
        Emax = self.scale(-1)
        log10Emax = int(math.log10(Emax)) + 1.0
        self.numberOfBin = int(log10Emax - LOG10_EMIN) * MESH_OF_BIN + 1
        nbin = self.numberOfBin
        e = np.array([10.0 ** (LOG10_EMIN + float(i) / float(MESH_OF_BIN)) for i in range(nbin)])
        self.binPos = np.zeros((nbin * self.nMat, 2), order="F")
        self.binNeg = np.zeros((nbin * self.nMat, 2), order="F")
        for m in range(self.nMat):
            self.binPos[m * nbin:(m + 1) * nbin, 0] = e
            self.binNeg[m * nbin:(m + 1) * nbin, 0] = -e
        self.numberOfBasis_old = self.nb            # main.F90:160
        self.ims_initial = None if self.ims is None else self.ims.copy()  # initialState.F90
        self.restore: Dict[int, dict] = {}
        self.thermo: Dict[int, tuple] = {}
        self.flow: Dict[int, np.ndarray] = {}
        self.ground_state_energy: Dict[int, float] = {}
        self.emin: Dict[int, float] = {}          # minimum before the shift (FDM energies)
        self.kept: Dict[int, int] = {}
        self.rdm_trace: Dict[int, float] = {}
        self.sum_warnings: List[tuple] = []
        self._full_init = False

    # --------------------------------------------------------------------------
    def _read_initial(self, path):
        toks = [ln.split() for ln in open(path).read().splitlines() if ln.strip()]
        it = iter(toks)
        nb, nVar, nCM, nC = self.nb, self.nVar, self.nCM, self.nCoef
        next(it)
        self.basis_output = np.zeros((nb, nVar + 3), dtype=np.int32)
        self.eigenvalue = np.zeros(nb)
        for i in range(nb):
            r = next(it)
            self.basis_output[i, :nVar + 1] = [int(x) for x in r[:nVar + 1]]
            self.eigenvalue[i] = _f(r[nVar + 1])
        next(it)
        self.im = np.zeros((nb, nb, nCM), order="F")
        for t in range(nCM):
            for j in range(nb):
                for k in range(nb):
                    self.im[k, j, t] = _f(next(it)[0])
        next(it)
        self.cim_type = np.zeros((nC, 3), dtype=np.int64)
        self.cim = np.zeros(nC)
        for i in range(nC):
            r = next(it)
            self.cim_type[i] = [int(x) for x in r[:3]]
            self.cim[i] = _f(r[3])
        next(it)
        self.cdiag_type = np.zeros((nC, 4), dtype=np.int64)
        self.cdiag = np.zeros(nC)
        for i in range(nC):
            r = next(it)
            self.cdiag_type[i] = [int(x) for x in r[:4]]
            self.cdiag[i] = _f(r[4])
        next(it)
        self.operation = np.zeros((self.nOps, nVar + self.nChain), dtype=np.int32)
        for i in range(self.nOps):
            self.operation[i] = [int(x) for x in next(it)[:nVar + self.nChain]]
        next(it)
        n = self.nIter + 2
        self.chain_diag = np.zeros((n, self.nChain))            # index 0..nIter+1
        self.chain_nond = np.zeros((n - self.first, self.nChain))  # first..nIter+1
        for c in range(self.nChain):
            next(it)
            for j in range(n):
                self.chain_diag[j, c] = _f(next(it)[0])
        for c in range(self.nChain):
            next(it)
            for j in range(n - self.first):
                self.chain_nond[j, c] = _f(next(it)[0])
        # rescale, read_initial_basis.F90:103-142 (ii = 0 .. nIter+1 only)
        L, z, D = self.Lambda, self.ztrick, self.bandWidth
        for c in range(self.nChain):
            for ii in range(0, n):
                if self.scalingType == 0:
                    fd, fn = L ** (float(ii - 1) * 0.5), L ** (float(ii) * 0.5)
                elif self.scalingType == 2:
                    fd = L ** (float(ii - 1) * 0.5 + z) * math.log(L) / D / (L - 1.0)
                    fn = L ** (float(ii) * 0.5 + z) * math.log(L) / D / (L - 1.0)
                else:
                    fd = L ** (float(ii - 1) * 0.5 + z - 1.0) / D * 2.0 / (1.0 + 1.0 / L)
                    fn = L ** (float(ii) * 0.5 + z - 1.0) / D * 2.0 / (1.0 + 1.0 / L)
                self.chain_diag[ii, c] = self.chain_diag[ii, c] * fd
                self.chain_nond[ii - self.first, c] = self.chain_nond[ii - self.first, c] * fn
        self.ims = None
        if self.flag_spectrum:
            nMat = self.nMat
            next(it)
            self.cspec = np.zeros((nMat, self.nOps))
            for m in range(nMat):
                for i in range(self.nOps):
                    self.cspec[m, i] = _f(next(it)[0])
            next(it)
            self.ims = np.zeros((nb, nb, nMat), order="F")
            for m in range(nMat):
                for j in range(nb):
                    for i in range(nb):
                        self.ims[i, j, m] = _f(next(it)[0])
            arrs = []
            for _ in range(3):
                next(it)
                a = np.zeros((nMat, nVar), dtype=np.int32)
                for m in range(nMat):
                    a[m] = [int(x) for x in next(it)[:nVar]]
                arrs.append(a)
            self.cons_diff, self.pos_op, self.neg_op = arrs
        if self.flag_BCS:
            self.chain_bcs = np.zeros((n, self.nChain))
            for c in range(self.nChain):
                next(it)
                for j in range(n):
                    self.chain_bcs[j, c] = _f(next(it)[0])
            next(it)
            self.coef_bcs = np.zeros((self.nBCS, 3), dtype=np.int64)
            for i in range(self.nBCS):
                self.coef_bcs[i] = [int(x) for x in next(it)[:3]]

    def scale(self, N: int) -> float:
        """module.F90:690-711"""
        L, z, D = self.Lambda, self.ztrick, self.bandWidth
        if self.scalingType == 0:
            return L ** (-float(N) * 0.5)
        if self.scalingType == 1:
            return D * 0.5 * (1.0 + 1.0 / L) * L ** (-float(N) * 0.5 - z + 1.0)
        return L ** (-float(N) * 0.5 - z) * D * (L - 1.0) / math.log(L)

    def cd(self, N, c):
        return self.chain_diag[N, c]

    def cn(self, N, c):
        return self.chain_nond[N - self.first, c]


# ------------------------------------------------------------------------------------
# coefficient lookups, restated as tables over (op_i, op_j)
# ------------------------------------------------------------------------------------
def diag_coef_table(st: State):
    """Outcome of the icoef loop of diagonalization.F90:195-213 per (op_i, op_j).

    Returns (flag, type, channel, coef, swapped); the last matching row wins for
    (type, channel, coef); ``swapped`` is set once any row matched in reversed order
    and is never reset inside the loop (the reference overwrites ireference/jreference
    only in the reversed branch).
    """
    n = st.nOps
    flag = np.zeros((n, n), dtype=bool)
    typ = np.zeros((n, n), dtype=np.int64)
    ch = np.zeros((n, n), dtype=np.int64)
    coef = np.zeros((n, n))
    swp = np.zeros((n, n), dtype=bool)
    for a in range(1, n + 1):
        for b in range(1, n + 1):
            for ic in range(st.nCoef):
                t = st.cdiag_type[ic]
                if a == t[0] and b == t[1]:
                    flag[a - 1, b - 1] = True
                    typ[a - 1, b - 1], ch[a - 1, b - 1] = t[2], t[3]
                    coef[a - 1, b - 1] = st.cdiag[ic]
                elif a == t[1] and b == t[0]:
                    flag[a - 1, b - 1] = True
                    typ[a - 1, b - 1], ch[a - 1, b - 1] = t[2], t[3]
                    coef[a - 1, b - 1] = st.cdiag[ic]
                    swp[a - 1, b - 1] = True
    return flag, typ, ch, coef, swp


def bcs_table(st: State):
    """diagonalization.F90:216-224: flag and (last) channel per (op_i, op_j)."""
    n = st.nOps
    flag = np.zeros((n, n), dtype=bool)
    ch = np.zeros((n, n), dtype=np.int64)
    if st.flag_BCS:
        for ic in range(st.nBCS):
            a, b, c = st.coef_bcs[ic]
            flag[a - 1, b - 1] = True
            ch[a - 1, b - 1] = c
    return flag, ch


def im_coef_table(st: State):
    """invariantMatrixDGEMM.F90:248-254: coefMatrix(i,j,type) = coef, last row wins."""
    n = st.nOps
    flag = np.zeros((n, n, st.nCM), dtype=bool)
    coef = np.zeros((n, n, st.nCM))
    for ic in range(st.nCoef):
        a, b, t = st.cim_type[ic]
        flag[a - 1, b - 1, t - 1] = True
        coef[a - 1, b - 1, t - 1] = st.cim[ic]
    return flag, coef


# ------------------------------------------------------------------------------------
# prepareBasis (prepareBasis.F90:31-114)
# ------------------------------------------------------------------------------------
def prepare_basis(st: State, iteration: int) -> None:
    nVar, nOps = st.nVar, st.nOps
    nb_old = st.numberOfBasis_old
    st.nb = nb_old * nOps                                     # :31
    bi = np.zeros((st.nb, nVar + 3), dtype=np.int32)
    pos = 0
    for i in range(nb_old):                                   # :42-57
        for j in range(nOps):
            bi[pos, :nVar] = st.basis_output[i, :nVar] - st.operation[j, :nVar]
            bi[pos, nVar] = i + 1
            bi[pos, nVar + 1] = st.basis_output[i, nVar]
            bi[pos, nVar + 2] = j + 1
            pos += 1
    exchange_sort(bi, nVar)                                   # :59
    st.basis_input = bi
    # sectors = runs of equal quantum numbers (:63-114)
    q = bi[:, :nVar]
    change = np.ones(st.nb, dtype=bool)
    change[1:] = np.any(q[1:] != q[:-1], axis=1)
    starts = np.nonzero(change)[0]
    dims = np.diff(np.append(starts, st.nb))
    nsub = len(starts)
    si = np.zeros((nsub, nVar + 3), dtype=np.int32)
    si[:, :nVar] = q[starts]
    si[:, nVar] = dims
    ce = np.ones(nsub, dtype=np.int64)
    ce[1:] = 1 + np.cumsum(dims[:-1].astype(np.int64) ** 2)
    si[:, nVar + 1] = ce          # count_eigenvector (int32 in the reference)
    si[:, nVar + 2] = starts + 1
    st.subspaceInfo = si
    st.numberOfSubspace = nsub


# ------------------------------------------------------------------------------------
# diagonalization (diagonalization.F90:1-410)
# ------------------------------------------------------------------------------------
def assemble_block(st: State, iteration: int, isub: int, tables=None) -> np.ndarray:
    """Sector Hamiltonian of diagonalization.F90:162-262 (full symmetric matrix)."""
    nVar = st.nVar
    if tables is None:
        tables = (diag_coef_table(st), bcs_table(st))
    (flag, typ, ch, coef, swp), (bflag, bch) = tables
    d = int(st.subspaceInfo[isub, nVar])
    s0 = int(st.subspaceInfo[isub, nVar + 2]) - 1
    rows = st.basis_input[s0:s0 + d]
    op = rows[:, nVar + 2].astype(np.int64) - 1
    ref = rows[:, nVar].astype(np.int64) - 1
    H = np.zeros((d, d))
    sq = math.sqrt(st.Lambda)
    diag = st.eigenvalue_prev[ref] * sq                                  # :285
    for c in range(st.nChain):                                          # :286-290
        diag = diag + st.operation[op, nVar + c].astype(np.float64) * st.cd(iteration + 1, c)
    H[np.arange(d), np.arange(d)] = diag
    if d > 1:
        iu, ju = np.triu_indices(d, 1)
        a, b = op[iu], op[ju]
        f = flag[a, b]
        sw = swp[a, b]
        ir = np.where(sw, ref[ju], ref[iu])
        jr = np.where(sw, ref[iu], ref[ju])
        tnd = np.array([st.cn(iteration, c) for c in range(st.nChain)])
        val = np.zeros(len(iu))
        if np.any(f):
            t_ = typ[a, b][f] - 1
            c_ = ch[a, b][f] - 1
            val[f] = (tnd[c_] * coef[a, b][f]) * st.im_prev[jr[f], ir[f], t_]   # :349-352
        if st.flag_BCS:
            bf = bflag[a, b] & (ir == jr)                                 # :336-342
            if np.any(bf):
                val[bf] = st.chain_bcs[iteration + 1, bch[a, b][bf] - 1]  # :359-364
        H[iu, ju] = val
        H[ju, iu] = val
    return H


def diagonalization(st: State, iteration: int) -> None:
    nVar = st.nVar
    tables = (diag_coef_table(st), bcs_table(st))
    dims = st.subspaceInfo[:, nVar].astype(np.int64)
    st.sizeOfEigenvector = int(np.sum(dims ** 2))
    ev = np.zeros(st.sizeOfEigenvector)
    E = np.zeros(st.nb)
    st.eigenvalue_prev = st.eigenvalue
    st.im_prev = st.im
    for isub in range(st.numberOfSubspace):
        d = int(dims[isub])
        H = assemble_block(st, iteration, isub, tables)
        w, V = scipy.linalg.eigh(H, lower=False, driver="ev", check_finite=False)  # :267
        V[np.abs(V) < EIGENVECTOR_THRESHOLD] = 0.0                        # :273-280
        s0 = int(st.subspaceInfo[isub, nVar + 2]) - 1
        c0 = int(st.subspaceInfo[isub, nVar + 1]) - 1
        E[s0:s0 + d] = w
        ev[c0:c0 + d * d] = V.ravel(order="F")
    st.ground_state_energy[iteration] = float(E[0])                       # :351
    st.emin[iteration] = float(np.min(E))
    E = E - np.min(E)                                                    # :353
    E[E <= NUMERICAL_THRESHOLD] = 0.0                                     # :354-356
    st.eigenvalue = E
    st.eigenvector = ev
    bo = np.zeros((st.nb, nVar + 3), dtype=np.int32)                      # :394-407
    for isub in range(st.numberOfSubspace):
        d = int(dims[isub])
        s0 = int(st.subspaceInfo[isub, nVar + 2]) - 1
        bo[s0:s0 + d, :nVar] = st.subspaceInfo[isub, :nVar]
        bo[s0:s0 + d, nVar] = np.arange(1, d + 1)
    st.basis_output = bo


# ------------------------------------------------------------------------------------
# postprocess (postprocess.F90:59-379) and thermodynamics (module.F90:1931-1982)
# ------------------------------------------------------------------------------------
def calc_thermo(st: State):
    Zn = En = Sz2n = Szn = 0.0
    s0, s1 = st.cb[1, 0], st.cb[1, 1]
    for i in range(st.nb):
        bE = BETABAR * st.eigenvalue[i]
        ex = math.exp(-bE)
        Zn += ex
        En += bE * ex
        Sz = int(np.sum(st.basis_output[i, s0 - 1:s1]))
        r = float(Sz) * 0.5
        Sz2n += ex * r * r
        Szn += ex * r
    Cn = 0.0
    for i in range(st.nb):
        bE = BETABAR * st.eigenvalue[i]
        ex = math.exp(-bE)
        Cn += (bE - En / Zn) * (bE - En / Zn) * ex
    Cn = Cn / Zn
    Sn = En / Zn + math.log(Zn)
    Xn = Sz2n / Zn - (Szn / Zn) * (Szn / Zn)
    return Cn, Sn, Xn


def truncate(st: State, iteration: int):
    """Sort and truncation of postprocess.F90:71-160.  Returns the kept count."""
    nb_full = st.nb
    st.numberOfBasis_full = nb_full
    idx = np.argsort(st.eigenvalue, kind="stable")           # sortWithIndex (:75), stable
    Es = st.eigenvalue[idx].copy()
    nb = nb_full
    if iteration != st.first and iteration != st.nIter and nb_full > st.truncation:
        if st.startTrancation > iteration:                   # :83-86
            st.startTrancation = iteration
            st.flag_truncation = True
        limit = int(st.truncation * TRUNCATION_LIMIT_SCALE)   # :87
        Ecut = Es[st.truncation - 1]
        i = st.truncation + 1
        cutoff = st.truncation
        Ecut = Ecut + TRUNCATION_THRESHOLD
        while i <= nb_full:
            if Es[i - 1] <= Ecut:
                cutoff += 1
            else:
                break
            i += 1
        while cutoff > limit:                                 # :109-123
            Ecut = Ecut - 0.001
            for i in range(cutoff, 0, -1):
                if Es[i - 1] > Ecut:
                    cutoff -= 1
                else:
                    break
        nb = cutoff
    st.flow[iteration] = Es[:nb].copy()
    # sortByIndex on the kept prefix (:140)
    order = np.argsort(idx[:nb], kind="stable")
    Es[:nb] = Es[:nb][order]
    idx[:nb] = idx[:nb][order]
    if nb < nb_full:                                         # :143-160
        st.basis_output = st.basis_output[idx].copy()
    st.eigenvalue = Es
    st.eigenindex = idx
    st.nb = nb
    st.kept[iteration] = nb
    return nb


def postprocess(st: State, iteration: int) -> None:
    st.thermo[iteration] = calc_thermo(st)                   # :62
    truncate(st, iteration)
    if iteration < st.nIter:                                 # :189-204
        invariant_matrix_dgemm(st, iteration)
        if st.flag_spectrum:
            invariant_matrix_for_spectrum_dgemm(st, iteration)
    st.numberOfBasis_old = st.nb                             # :207
    if st.flag_spectrum:
        store_restore(st, iteration)                         # :212-217
        if iteration >= st.startTrancation:
            stock_full(st, iteration)                        # :221-374


def keeped_basis_number(st: State) -> np.ndarray:
    """invariantMatrixDGEMM.F90:84-100: kept states per sector."""
    nVar = st.nVar
    kb = np.zeros(st.numberOfSubspace, dtype=np.int64)
    kept_q = st.basis_output[:st.nb, :nVar]
    for isub in range(st.numberOfSubspace):
        kb[isub] = int(np.sum(np.all(kept_q == st.subspaceInfo[isub, :nVar], axis=1)))
    return kb


def _vectors(st: State, isub: int, ncol: int, first_col: int = 0) -> np.ndarray:
    """Columns first_col .. first_col+ncol-1 of the eigenvector block of sector isub
    (column semantics of invariantMatrixDGEMM.F90:222-228)."""
    nVar = st.nVar
    d = int(st.subspaceInfo[isub, nVar])
    c0 = int(st.subspaceInfo[isub, nVar + 1]) - 1
    blk = st.eigenvector[c0:c0 + d * d].reshape((d, d), order="F")
    return blk[:, first_col:first_col + ncol]


def invariant_matrix_dgemm(st: State, iteration: int) -> None:
    """invariantMatrixDGEMM.F90:67-341 (single rank: no ALLREDUCE)."""
    nVar = st.nVar
    nb = st.nb
    im = np.zeros((nb, nb, st.nCM), order="F")
    cs, ce_ = st.cb[0, 0], st.cb[0, 1]
    ss, se = st.cb[1, 0], st.cb[1, 1]
    kb = keeped_basis_number(st)
    kstart = np.concatenate([[0], np.cumsum(kb)])
    flag, coef = im_coef_table(st)
    si = st.subspaceInfo
    for il in range(st.numberOfSubspace):
        for ir in range(st.numberOfSubspace):
            if kb[il] == 0 or kb[ir] == 0:
                continue
            dq = si[il, :nVar].astype(np.int64) - si[ir, :nVar]
            if cs == ce_ and cs == 0:                                   # :170-178
                dS = int(np.sum(dq[ss - 1:se]))
                if abs(dS) != 1:
                    continue
            else:
                dQ = int(np.sum(dq[cs - 1:ce_]))
                dS = int(np.sum(dq[ss - 1:se]))
                if dQ != 1 or abs(dS) != 1:
                    continue
            dL, dR = int(si[il, nVar]), int(si[ir, nVar])
            bL, bR = int(si[il, nVar + 2]) - 1, int(si[ir, nVar + 2]) - 1
            VL = _vectors(st, il, int(kb[il]))           # (dL, kL); vectorL = VL^T
            VR = _vectors(st, ir, int(kb[ir]))           # (dR, kR)
            varL = st.basis_input[bL:bL + dL, nVar + 1]
            varR = st.basis_input[bR:bR + dR, nVar + 1]
            opL = st.basis_input[bL:bL + dL, nVar + 2] - 1
            opR = st.basis_input[bR:bR + dR, nVar + 2] - 1
            same_var = varL[:, None] == varR[None, :]                  # :243-245
            for t in range(st.nCM):                                    # :284
                C = np.where(same_var & flag[opL[:, None], opR[None, :], t],
                             coef[opL[:, None], opR[None, :], t], 0.0)
                tmp1 = VL.T @ C                                        # :300
                sub = tmp1 @ VR                                        # :316
                sl, sr = kstart[il], kstart[ir]
                im[sr:sr + kb[ir], sl:sl + kb[il], t] = sub.T          # :327-332
    st.im = im


def _ims_coef_matrix(st, bL, dL, bR, dR, m, ims):
    """coefMatrix of invariantMatrixForSpectrumDGEMM.F90:235-256 / module.F90:1070-1091."""
    nVar = st.nVar
    opL = st.basis_input[bL:bL + dL, nVar + 2] - 1
    opR = st.basis_input[bR:bR + dR, nVar + 2] - 1
    refL = st.basis_input[bL:bL + dL, nVar] - 1
    refR = st.basis_input[bR:bR + dR, nVar] - 1
    same = opL[:, None] == opR[None, :]
    vals = st.cspec[m, opL][:, None] * ims[refR[None, :], refL[:, None], m]
    return np.where(same, vals, 0.0)


def invariant_matrix_for_spectrum_dgemm(st: State, iteration: int) -> None:
    """invariantMatrixForSpectrumDGEMM.F90:71-370 (single rank)."""
    nVar = st.nVar
    nb = st.nb
    new = np.zeros((nb, nb, st.nMat), order="F")
    kb = keeped_basis_number(st)
    kstart = np.concatenate([[0], np.cumsum(kb)])
    si = st.subspaceInfo
    ims_prev = st.ims
    for il in range(st.numberOfSubspace):
        for ir in range(st.numberOfSubspace):
            if kb[il] == 0 or kb[ir] == 0:
                continue
            diff = si[il, :nVar].astype(np.int64) - si[ir, :nVar]          # :166
            mats = [m for m in range(st.nMat) if np.all(diff == st.cons_diff[m])]
            if not mats:
                continue
            dL, dR = int(si[il, nVar]), int(si[ir, nVar])
            bL, bR = int(si[il, nVar + 2]) - 1, int(si[ir, nVar + 2]) - 1
            VL = _vectors(st, il, int(kb[il]))
            VR = _vectors(st, ir, int(kb[ir]))
            for m in mats:
                C = _ims_coef_matrix(st, bL, dL, bR, dR, m, ims_prev)
                sub = (VL.T @ C) @ VR                                     # :296-313
                sl, sr = kstart[il], kstart[ir]
                new[sr:sr + kb[ir], sl:sl + kb[il], m] = sub.T            # :323-328
    st.ims = new


def store_restore(st: State, iteration: int) -> None:
    """initRestore / appendRestore (module.F90:1345-1570): per-iteration copies."""
    rec = dict(
        eigenvalue=st.eigenvalue.copy(), eigenvector=st.eigenvector.copy(),
        basis_output=st.basis_output.copy(), basis_input=st.basis_input.copy(),
        subspaceInfo=st.subspaceInfo.copy(), numberOfBasis=st.nb,
        numberOfBasis_full=st.numberOfBasis_full, ims=None,
    )
    if iteration == st.first or iteration < st.nIter:
        rec["ims"] = st.ims.copy()
    st.restore[iteration] = rec


def stock_full(st: State, iteration: int) -> None:
    """postprocess.F90:221-374: the "full" stock used by the RDM and the CFS spectrum."""
    nVar = st.nVar
    if not st._full_init:                                     # :228-249
        st._full_init = True
        st.pointFullBasisInput = 1
        st.pointFullBasisOutput = 1
        st.pointFullEigenvector = 1
        st.pointFullSubspace = 1
        st.mapFull = {}
        st.fullSubspaceInfo = []
        st.fullBasisInput = []
        st.fullBasisOutput = []
        st.fullEigenvalue = []
        st.fullEigenvector = []
        st.sizeOfReducedDensity = 0
    st.mapFull[iteration] = st.pointFullSubspace              # :236, :290
    st.fullBasisOutput.append(st.basis_output[:st.nb].copy())  # :294-297
    st.fullEigenvalue.append(st.eigenvalue[:st.nb].copy())
    st.fullBasisInput.append(st.basis_input[:st.numberOfBasis_full].copy())  # :299-301
    kept_q = st.basis_output[:st.nb, :nVar]
    for i in range(st.numberOfSubspace):                      # :303-368
        match = np.nonzero(np.all(kept_q == st.subspaceInfo[i, :nVar], axis=1))[0]
        k = len(match)
        if k > 0:
            d = int(st.subspaceInfo[i, nVar])
            row = np.zeros(nVar + 6, dtype=np.int64)
            row[:nVar] = st.subspaceInfo[i, :nVar]
            row[nVar] = d
            row[nVar + 1] = k
            row[nVar + 2] = st.pointFullEigenvector
            row[nVar + 3] = st.pointFullBasisInput + int(st.subspaceInfo[i, nVar + 2]) - 1
            row[nVar + 4] = st.pointFullBasisOutput + int(match[0])
            row[nVar + 5] = 0
            st.sizeOfReducedDensity += k * k
            c0 = int(st.subspaceInfo[i, nVar + 1]) - 1
            st.fullEigenvector.append(st.eigenvector[c0:c0 + d * k].copy())
            st.pointFullEigenvector += d * k
            st.fullSubspaceInfo.append(row)
            st.pointFullSubspace += 1
    st.pointFullBasisInput += st.numberOfBasis_full
    st.pointFullBasisOutput += st.nb


def nrg_iteration(st: State, iteration: int) -> None:
    """nrgIteration.F90:1-31 (loadbalance is a no-op on one process)."""
    prepare_basis(st, iteration)
    diagonalization(st, iteration)
    postprocess(st, iteration)


# ------------------------------------------------------------------------------------
# reduced density matrix (initializeReducedDensity.F90, reducedDensityMatrixDGEMM.F90)
# ------------------------------------------------------------------------------------
def _finalize_full(st: State) -> None:
    st.FSI = np.array(st.fullSubspaceInfo, dtype=np.int64).reshape(-1, st.nVar + 6)
    st.FBI = np.concatenate(st.fullBasisInput)
    st.FBO = np.concatenate(st.fullBasisOutput)
    st.FE = np.concatenate(st.fullEigenvalue)
    st.FV = np.concatenate(st.fullEigenvector) if st.fullEigenvector else np.zeros(0)
    st.elementNumFullSubspace = st.pointFullSubspace - 1


def initialize_reduced_density(st: State) -> None:
    """initializeReducedDensity.F90:32-78 (T = 0: projector on the ground states)."""
    nVar = st.nVar
    _finalize_full(st)
    deg = int(np.sum(st.eigenvalue[:st.nb] < DEGENERACY_THRESHOLD))
    pf = float(deg)
    st.rdm = np.zeros(st.sizeOfReducedDensity)
    idx0 = st.mapFull[st.nIter] - 1
    point = 1
    for i in range(st.numberOfSubspace):
        row = st.FSI[idx0 + i]
        row[nVar + 5] = point
        k = int(row[nVar + 1])
        for a in range(k):
            for b in range(k):
                if a == b:
                    e = st.FE[int(row[nVar + 4]) - 1 + a]
                    if e < DEGENERACY_THRESHOLD:
                        st.rdm[point - 1] = 1.0 / pf
                point += 1
    st.pointReducedDensity = point


def reduced_density_matrix_calculation(st: State) -> None:
    """reducedDensityMatrixDGEMM.F90:62-372 (single rank)."""
    nVar, nOps = st.nVar, st.nOps
    if not st.flag_truncation:
        return
    FSI = st.FSI
    for i in range(1, st.nIter - st.startTrancation + 1):
        present = st.nIter - i
        previous = present + 1
        ps = st.mapFull[present] - 1
        qs = st.mapFull[previous] - 1
        for j in range(ps, qs):                                   # :94-100
            FSI[j, nVar + 5] = st.pointReducedDensity
            st.pointReducedDensity += int(FSI[j, nVar + 1]) ** 2
        if previous == st.nIter:                                  # :177-182
            q_end = st.elementNumFullSubspace - 1
        else:
            q_end = st.mapFull[previous + 1] - 2
        diag = 0.0
        for iS in range(ps, qs):
            qn = FSI[iS, :nVar]
            n = int(FSI[iS, nVar + 1])
            pout = int(FSI[iS, nVar + 4]) - 1
            found = []
            for op in range(nOps):                                # :164-204
                pq = qn - st.operation[op, :nVar]
                hit = None
                for iSp in range(qs, q_end + 1):
                    if np.all(FSI[iSp, :nVar] == pq):
                        hit = iSp
                found.append(hit)
            keep = [0 if h is None else int(FSI[h, nVar + 1]) for h in found]
            T = sum(keep)
            rho_prev = np.zeros((T, T))
            A = np.zeros((n, T))
            startl = 0
            for op in range(nOps):                                # :224-260
                h = found[op]
                if h is not None:
                    k = keep[op]
                    dprev = int(FSI[h, nVar])
                    pe = int(FSI[h, nVar + 2]) - 1
                    pi = int(FSI[h, nVar + 3]) - 1
                    pm = int(FSI[h, nVar + 5]) - 1
                    rho_prev[startl:startl + k, startl:startl + k] = \
                        st.rdm[pm:pm + k * k].reshape((k, k))       # row-major, :230-234
                    var = st.FBI[pi:pi + dprev, nVar + 1]
                    opr = st.FBI[pi:pi + dprev, nVar + 2]
                    for il in range(n):
                        present_index = st.FBO[pout + il, nVar]   # :239
                        hits = np.nonzero((var == present_index) & (opr == op + 1))[0]
                        assert len(hits) > 0, "no derived state (reference would reuse a stale index)"
                        ild = int(hits[0])
                        A[il, startl:startl + k] = st.FV[pe + ild: pe + ild + k * dprev: dprev]
                startl += keep[op]
            tmp1 = A @ rho_prev                                   # :280
            rs = tmp1 @ A.T                                       # :296
            diag += float(np.trace(rs))
            pm = int(FSI[iS, nVar + 5]) - 1
            st.rdm[pm:pm + n * n] = rs.reshape(-1)                 # row-major, :308-314
        st.rdm_trace[present] = diag


# ------------------------------------------------------------------------------------
# CFS spectrum (module.F90:1014-1338, 1573-1706; calculateSpectrumDGEMM.F90)
# ------------------------------------------------------------------------------------
def get_restore(st: State, iteration: int) -> dict:
    """getRestore (module.F90:1573-1681)."""
    r = st.restore[iteration]
    ims = st.restore[iteration - 1]["ims"] if iteration > st.first else st.ims_initial
    return dict(r, ims_prev=ims, nb_old=(st.restore[iteration - 1]["numberOfBasis"]
                                         if iteration > st.first else None))


def bin_spikes(st: State, container: np.ndarray, energy: np.ndarray, weight: np.ndarray,
               m: int) -> None:
    """binningSpike (module.F90:1210-1254), vectorised over spikes in order."""
    nbin = st.numberOfBin
    with np.errstate(divide="ignore"):
        position = (np.log10(np.abs(energy)) - LOG10_EMIN) * MESH_OF_BIN + 1.0
    pr = np.trunc(position)
    pr = np.where(np.isfinite(pr), pr, 0.0).astype(np.int64)
    lo = position <= 0.0
    hi = (~lo) & (position >= nbin)
    pr = np.where(pr <= 0, 1, pr)
    one = lo | hi
    i1 = np.where(lo, 1, np.where(hi, nbin, pr))
    wb = position - pr.astype(np.float64)
    off = m * nbin - 1
    # same-bin spikes: all weight to i1
    idx_a = np.where(one, i1, pr) + off
    with np.errstate(invalid="ignore"):   # wb is NaN at E = 0, where the one-bin branch is taken
        w_a = np.where(one, weight, weight * (1.0 - wb))
    np.add.at(container[:, 1], idx_a, w_a)
    two = ~one
    if np.any(two):
        np.add.at(container[:, 1], pr[two] + 1 + off, weight[two] * wb[two])


def log_grid(wmin: float = 1e-8, wmax: float = 1.0, per_decade: int = 100) -> np.ndarray:
    """Positive frequencies wmin .. wmax, per_decade points per decade (both ends kept)."""
    n = int(round(np.log10(wmax / wmin) * per_decade))
    return wmin * 10.0 ** (np.arange(n + 1) / per_decade)


def broaden_log_gaussian(bins: np.ndarray, nbin: int, nmat: int, b: float, omega: np.ndarray) -> np.ndarray:
    """Log-Gaussian broadening of binned spikes (Bulla, Costi and Pruschke, Rev. Mod. Phys.
    80, 395 (2008), Sec. V.A; the reference has none: it writes raw bins):
    A_m(w) = sum_i w_i exp(-b^2/4) / (b |E_i| sqrt(pi)) exp(-(ln(w/E_i)/b)^2), w E_i > 0.
    bins: (nbin*nmat, 2) energies and weights as spikeCFS fills them.  Returns (nmat, len(w))."""
    omega = np.asarray(omega, dtype=np.float64)
    out = np.zeros((nmat, omega.size))
    pref = math.exp(-0.25 * b * b) / (b * math.sqrt(math.pi))
    for m in range(nmat):
        E = bins[m * nbin:(m + 1) * nbin, 0]
        W = bins[m * nbin:(m + 1) * nbin, 1]
        nz = W != 0.0
        E, W = E[nz], W[nz]
        for k, w in enumerate(omega):
            same = w * E > 0.0
            if not np.any(same):
                continue
            x = np.log(w / E[same]) / b
            out[m, k] = pref * np.sum(W[same] * np.exp(-x * x) / np.abs(E[same]))
    return out


def _find_subspace(si, nVar, qn):
    """findSubspace (module.F90:1256-1284): first match."""
    hit = np.nonzero(np.all(si[:, :nVar] == qn, axis=1))[0]
    return int(hit[0]) if len(hit) else None


def spectrum_element_dgemm(st, R, isub_left, dim_left, col_left, isub_right, dim_right,
                           col_right, m):
    """spectrumElementDGEMM (module.F90:1014-1125) with column semantics."""
    nVar = st.nVar
    si = R["subspaceInfo"]

    def block(isub, ncol, c0):
        d = int(si[isub, nVar])
        e0 = int(si[isub, nVar + 1]) - 1
        return R["eigenvector"][e0:e0 + d * d].reshape((d, d), order="F")[:, c0:c0 + ncol]

    dL, dR = int(si[isub_left, nVar]), int(si[isub_right, nVar])
    bL, bR = int(si[isub_left, nVar + 2]) - 1, int(si[isub_right, nVar + 2]) - 1
    VL = block(isub_left, dim_left, col_left)
    VR = block(isub_right, dim_right, col_right)
    bi = R["basis_input"]
    opL = bi[bL:bL + dL, nVar + 2] - 1
    opR = bi[bR:bR + dR, nVar + 2] - 1
    refL = bi[bL:bL + dL, nVar] - 1
    refR = bi[bR:bR + dR, nVar] - 1
    ims = R["ims_prev"]
    C = np.where(opL[:, None] == opR[None, :],
                 st.cspec[m, opL][:, None] * ims[refR[None, :], refL[:, None], m], 0.0)
    return (VL.T @ C) @ VR


def spike_zero_temperature(st: State, iteration: int, R: Optional[dict] = None) -> None:
    """calculateSpectrumDGEMM.F90:1-215 (raw spike files are not written)."""
    nVar = st.nVar
    if R is None:
        R = get_restore(st, iteration)
    E = R["eigenvalue"]
    bo = R["basis_output"]
    si = R["subspaceInfo"]
    nb = R["numberOfBasis"]
    gs = np.nonzero(E[:nb] < DEGENERACY_THRESHOLD)[0]                    # :56-75
    pf = float(len(gs))
    sc = st.scale(iteration)
    for g in gs:
        qg = bo[g, :nVar].astype(np.int64)
        isg = _find_subspace(si, nVar, qg)
        for sign, opsarr, cont in ((+1, st.pos_op, st.binPos), (-1, st.neg_op, st.binNeg)):
            for m in range(st.nMat):
                qe = qg + opsarr[m]
                ise = _find_subspace(si, nVar, qe)
                if ise is None:
                    continue
                dE = int(si[ise, nVar])
                b0 = int(si[ise, nVar + 2]) - 1
                if sign > 0:   # <ex|d^dag|g>, GS column 1 always (:107-111)
                    s = spectrum_element_dgemm(st, R, ise, dE, 0, isg, 1, 0, m)[:, 0]
                else:          # <g|d^dag|ex>
                    s = spectrum_element_dgemm(st, R, isg, 1, 0, ise, dE, 0, m)[0, :]
                en = sign * E[b0:b0 + dE] * sc
                w = s * s / pf
                bin_spikes(st, cont, en, w, m)


def spike_cfs(st: State, iteration: int, nb_full: int, R: Optional[dict] = None,
              literal: bool = False) -> None:
    """calculateSpectrumDGEMM.F90:217-646 (single rank).

    ``literal=True`` loops over discarded states one at a time exactly like the
    reference; the default batches the discarded states of one sector into one product
    (the same per-column arithmetic).
    """
    nVar = st.nVar
    if R is None:
        R = get_restore(st, iteration)
    E = R["eigenvalue"]
    bo = R["basis_output"]
    si = R["subspaceInfo"]
    nb = R["numberOfBasis"]
    sc = st.scale(iteration)
    nbin = st.numberOfBin
    tmpPos = np.zeros((nbin * st.nMat, 2), order="F")
    tmpNeg = np.zeros((nbin * st.nMat, 2), order="F")
    tot_pos = np.zeros(st.nMat)
    tot_neg = np.zeros(st.nMat)
    FSI = st.FSI
    f0 = st.mapFull[iteration] - 1
    f1 = st.mapFull[iteration + 1] - 1

    def find_full(q):
        hit = np.nonzero(np.all(FSI[f0:f1, :nVar] == q, axis=1))[0]
        return f0 + int(hit[0]) if len(hit) else None

    def start_output(q):    # findStartOutput (module.F90:1316-1338)
        hit = np.nonzero(np.all(bo[:nb, :nVar] == q, axis=1))[0]
        return int(hit[0])

    # discarded states nb+1 .. nb_full (:363-368), one at a time (literal) or grouped by
    # sector (same per-column arithmetic)
    items = [(_find_subspace(si, nVar, bo[il, :nVar]), [il]) for il in range(nb, nb_full)]
    if not literal:
        groups: Dict[int, List[int]] = {}
        for isl, ls in items:
            groups.setdefault(isl, []).extend(ls)
        items = list(groups.items())
    for isl, ls in items:
        ls = np.array(ls)
        ql = si[isl, :nVar].astype(np.int64)
        cols = bo[ls, nVar] - 1
        El = E[ls]
        dl = int(si[isl, nVar])
        e0 = int(si[isl, nVar + 1]) - 1
        Vl = R["eigenvector"][e0:e0 + dl * dl].reshape((dl, dl), order="F")[:, cols]
        for part in (0, 1):
            opsarr = st.pos_op if part == 0 else st.neg_op
            for m in range(st.nMat):
                qk = ql + opsarr[m]
                fk = find_full(qk)
                isk = _find_subspace(si, nVar, qk)
                if fk is None or isk is None:
                    continue
                sbo = start_output(qk)
                kk = int(FSI[fk, nVar + 1])
                pm = int(FSI[fk, nVar + 5]) - 1
                assert int(FSI[fk, nVar]) == int(si[isk, nVar])   # :418-423
                # rho(k2, k1) read as reducedDensityMatrix(pm + kk*(k2-1) + (k1-1))
                k1v = bo[sbo:sbo + kk, nVar] - 1
                rho = st.rdm[pm:pm + kk * kk]
                X = rho[kk * k1v[None, :] + k1v[:, None]]          # X[k1, k2] = rho(k2,k1)
                # part 0: S(k1, l) = <k1|d^dag|l> (:429-432); part 1: <l|d^dag|k1> (:508-511)
                S = _spec_batch(st, R, isk, kk, isl, Vl, m, left_is_k=(part == 0))
                # S: (kk, nl); w(k1, l) = sum_k2 S(k1) S(k2) rho(k2,k1)
                W = S * (X @ S)
                Ek = E[sbo:sbo + kk]
                if part == 0:
                    en = (Ek[:, None] - El[None, :]) * sc           # :442
                    cont, tot = tmpNeg, tot_neg
                else:
                    en = (El[None, :] - Ek[:, None]) * sc           # :519
                    cont, tot = tmpPos, tot_pos
                tot[m] += float(np.sum(W))
                bin_spikes(st, cont, en.T.reshape(-1), W.T.reshape(-1), m)
    # :559-596 binned vs raw sums
    for m in range(st.nMat):
        for cont, tot, name in ((tmpNeg, tot_neg, "negative"), (tmpPos, tot_pos, "positive")):
            sb = float(np.sum(cont[m * nbin:(m + 1) * nbin, 1]))
            if abs(sb - tot[m]) >= DEGENERACY_THRESHOLD:
                st.sum_warnings.append((iteration, name, m + 1, sb - tot[m]))
    st.binNeg[:, 1] += tmpNeg[:, 1]                                     # :627-643
    st.binPos[:, 1] += tmpPos[:, 1]


def _spec_batch(st, R, isk, kk, isl, Vl, m, left_is_k):
    """spectrumElementDGEMM for all columns of Vl at once; returns (kk, n_l)."""
    nVar = st.nVar
    si = R["subspaceInfo"]
    dk = int(si[isk, nVar])
    ek = int(si[isk, nVar + 1]) - 1
    Vk = R["eigenvector"][ek:ek + dk * dk].reshape((dk, dk), order="F")[:, :kk]
    bi = R["basis_input"]
    bK = int(si[isk, nVar + 2]) - 1
    bL = int(si[isl, nVar + 2]) - 1
    dl = int(si[isl, nVar])
    ims = R["ims_prev"]
    if left_is_k:
        C = _coef(st, bi, bK, dk, bL, dl, m, ims)
        return (Vk.T @ C) @ Vl
    C = _coef(st, bi, bL, dl, bK, dk, m, ims)
    return ((Vl.T @ C) @ Vk).T


def _coef(st, bi, bL, dL, bR, dR, m, ims):
    nVar = st.nVar
    opL = bi[bL:bL + dL, nVar + 2] - 1
    opR = bi[bR:bR + dR, nVar + 2] - 1
    refL = bi[bL:bL + dL, nVar] - 1
    refR = bi[bR:bR + dR, nVar] - 1
    return np.where(opL[:, None] == opR[None, :],
                    st.cspec[m, opL][:, None] * ims[refR[None, :], refL[:, None], m], 0.0)


def cfs_spectrum_calculation(st: State, iteration: int, literal: bool = False) -> None:
    """cfsSpectrumCalculation (module.F90:1683-1706)."""
    R = get_restore(st, iteration)
    if iteration == st.nIter:
        spike_zero_temperature(st, iteration, R)
    else:
        spike_cfs(st, iteration, R["numberOfBasis_full"], R, literal=literal)


# ------------------------------------------------------------------------------------
# driver (main.F90:142-252)
# ------------------------------------------------------------------------------------
def run(directory: str, spectrum: bool = True, literal: bool = False,
        stop_after: Optional[int] = None) -> State:
    st = State(directory)
    last = st.nIter if stop_after is None else stop_after
    for it in range(st.first, last + 1):                      # main.F90:175-177
        nrg_iteration(st, it)
    if spectrum and st.flag_spectrum and stop_after is None:
        if st.flag_truncation:                                # main.F90:188-201
            initialize_reduced_density(st)
            reduced_density_matrix_calculation(st)
        for it in range(st.startTrancation, st.nIter + 1):    # main.F90:204-224
            cfs_spectrum_calculation(st, it, literal=literal)
    return st


# ------------------------------------------------------------------------------------
# restart.dat of the CFS phase (module.F90:1710-1890; main.F90:165-224)
# ------------------------------------------------------------------------------------
MODE_RESTART_NON = 1000            # module.F90:1718
MODE_RESTART_CFS = 1002            # module.F90:1720
_RESTORE_FIELDS = 10               # type restore, module.F90:983-994


def _hami_words(st: State, numberOfBasis: int) -> np.ndarray:
    """HamiltonianInfo_type (module.F90:722-760) as written by ``write(fd) hami``: its
    components in order, 4-byte integers and logicals (.true. = 1)."""
    cb = st.cb.ravel(order="F")
    return np.array([st.nIter, st.nChain, st.nVar, cb[0], cb[1], cb[2], cb[3], st.nMat, st.nCM,
                     numberOfBasis, st.nCoef, 0, st.nOps, st.nBCS, st.first, int(st.flag_spectrum), 0,
                     st.startTrancation, int(st.flag_truncation), int(st.flag_BCS)], dtype="<i4")


def save_restart(st: State, iteration: int, path: str, numberOfBasis: int) -> None:
    """saveRestart (module.F90:1723-1785): Fortran stream output (no record markers).
    ``numberOfBasis`` is hami%numberOfBasis at the call (the kept count of the last
    iteration before the first CFS step, that of iteration-1 after getRestore)."""
    its = range(st.first, st.nIter + 1)
    ri = np.zeros((st.nIter + 2 - st.first, _RESTORE_FIELDS), dtype=np.int64)
    e0 = v0 = s0 = m0 = 1
    for x, it in enumerate(its):                      # initRestore/appendRestore :1388-1567
        r = st.restore[it]
        nf, nv, ns, nb = r["numberOfBasis_full"], r["eigenvector"].size, len(r["subspaceInfo"]), r["numberOfBasis"]
        nm = nb * nb * st.nMat if it < st.nIter else 0
        ri[x] = [e0, nf, v0, nv, s0, ns, e0, m0 if nm else 0, nm, nb]
        e0, v0, s0, m0 = e0 + nf, v0 + nv, s0 + ns, m0 + nm

    def i4(a):
        return np.ascontiguousarray(a, dtype="<i4").tobytes()

    def f8(a):
        return np.ascontiguousarray(a, dtype="<f8").tobytes()

    R = [st.restore[it] for it in its]
    with open(path, "wb") as f:
        f.write(i4([MODE_RESTART_CFS, iteration]))
        f.write(_hami_words(st, numberOfBasis).tobytes())
        f.write(i4([st.first, st.nIter + 1]) + i4(ri.ravel()))
        for key in ("subspaceInfo", "basis_input", "basis_output"):
            recs = [r[key][:r["numberOfBasis_full"]] if key != "subspaceInfo" else r[key] for r in R]
            f.write(i4([sum(len(a) for a in recs)]))
            for a in recs:
                f.write(i4(a))
        ims = [r["ims"].ravel(order="F") for it, r in zip(its, R) if it < st.nIter]
        f.write(i4([sum(a.size for a in ims)]))
        for a in ims:
            f.write(f8(a))
        f.write(i4(list(st.ims_initial.shape)) + f8(st.ims_initial.ravel(order="F")))
        f.write(i4([sum(r["numberOfBasis_full"] for r in R)]))
        for r in R:
            f.write(f8(r["eigenvalue"][:r["numberOfBasis_full"]]))
        f.write(i4([sum(r["eigenvector"].size for r in R)]))
        for r in R:
            f.write(f8(r["eigenvector"]))
        f.write(i4([st.rdm.size]) + f8(st.rdm))
        f.write(i4([len(st.FSI)]) + i4(st.FSI))
        mp = np.zeros(st.nIter + 2, dtype=np.int64)
        for it, v in st.mapFull.items():
            mp[it + 1] = v
        f.write(i4([-1, st.nIter]) + i4(mp))
        for b in (st.binPos, st.binNeg):
            f.write(i4([b.size]) + f8(b.ravel(order="F")))


def load_restart(st: State, path: str) -> int:
    """loadRestart (module.F90:1787-1890): the restore and full stocks, the density
    matrices and the bins; returns iteration_restart."""
    buf = open(path, "rb").read()
    pos = 0

    def take(n, dt):
        nonlocal pos
        a = np.frombuffer(buf, dtype=dt, count=n, offset=pos)
        pos += a.nbytes
        return a

    def i4(n=1):
        return take(n, "<i4").astype(np.int64)

    mode, iteration = (int(x) for x in i4(2))
    if mode != MODE_RESTART_CFS:
        raise ValueError("broken restart file")
    h = i4(20)
    st.startTrancation, st.flag_truncation = int(h[17]), bool(h[18])
    lo, hi = (int(x) for x in i4(2))
    ri = i4((hi - lo + 1) * _RESTORE_FIELDS).reshape(-1, _RESTORE_FIELDS)
    rs, rsf = st.nVar + 3, st.nVar + 6
    arrays = {}
    for key in ("subspaceInfo", "basis_input", "basis_output"):
        n = int(i4()[0])
        arrays[key] = i4(n * rs).reshape(n, rs)
    ims = take(int(i4()[0]), "<f8")
    d = [int(x) for x in i4(3)]
    st.ims_initial = take(d[0] * d[1] * d[2], "<f8").reshape(d, order="F").copy()
    E = take(int(i4()[0]), "<f8")
    V = take(int(i4()[0]), "<f8")
    st.rdm = take(int(i4()[0]), "<f8").copy()
    n = int(i4()[0])
    st.FSI = i4(n * rsf).reshape(n, rsf)
    st.elementNumFullSubspace = n
    lo, hi = (int(x) for x in i4(2))
    mp = i4(hi - lo + 1)
    st.mapFull = {it: int(mp[it - lo]) for it in range(lo, hi + 1) if mp[it - lo] != 0}
    for name in ("binPos", "binNeg"):
        n = int(i4()[0])
        setattr(st, name, take(n, "<f8").reshape((n // 2, 2), order="F").copy())
    assert pos == len(buf), "trailing bytes in the restart file"
    st.restore = {}
    for x, it in enumerate(range(st.first, st.nIter + 1)):     # getRestore :1596-1660
        e, nf, v, nv, s, ns, b, m, nm, nb = (int(q) for q in ri[x])
        st.restore[it] = dict(
            eigenvalue=E[e - 1:e - 1 + nf].copy(), eigenvector=V[v - 1:v - 1 + nv].copy(),
            basis_output=arrays["basis_output"][b - 1:b - 1 + nf].copy(),
            basis_input=arrays["basis_input"][b - 1:b - 1 + nf].copy(),
            subspaceInfo=arrays["subspaceInfo"][s - 1:s - 1 + ns].copy(), numberOfBasis=nb,
            numberOfBasis_full=nf,
            ims=(ims[m - 1:m - 1 + nm].reshape((nb, nb, st.nMat), order="F").copy() if nm else None))
    return iteration


def run_with_restart(directory: str, save_path: Optional[str] = None, load_path: Optional[str] = None,
                     stop_before: Optional[int] = None) -> State:
    """main.F90:160-224 with param%saveRestart (``save_path``) and param%loadRestart
    (``load_path``).  ``stop_before`` ends the run right after the file was written for
    that CFS step, as an interrupted job would leave it."""
    st = State(directory)
    mode = MODE_RESTART_NON
    it_r = None
    if load_path:
        it_r = load_restart(st, load_path)
        mode = MODE_RESTART_CFS
    if mode != MODE_RESTART_CFS:
        for it in range(st.first, st.nIter + 1):
            nrg_iteration(st, it)
        if st.flag_truncation:
            initialize_reduced_density(st)
            reduced_density_matrix_calculation(st)
    first_step = True
    for it in range(st.startTrancation, st.nIter + 1):
        if mode == MODE_RESTART_CFS and it < it_r:
            continue
        if save_path and (mode != MODE_RESTART_CFS or it > it_r):
            nb = st.restore[st.nIter]["numberOfBasis"] if (first_step and mode != MODE_RESTART_CFS) \
                else st.restore[it - 1]["numberOfBasis"]
            save_restart(st, it, save_path, nb)
        first_step = False
        if stop_before is not None and it == stop_before:
            return st
        cfs_spectrum_calculation(st, it)
    return st


# ------------------------------------------------------------------------------------
# full-density-matrix (FDM) spectrum at temperature T.  The reference has none (its
# spectrum is the T = 0 CFS one); restated from the published method: Weichselbaum and
# von Delft, PRL 99, 076402 (2007), with the complete basis of Anders and Schiller, PRL
# 95, 196801 (2005).
# ------------------------------------------------------------------------------------
def _shell(st: State, N: int) -> dict:
    """Shell N from the restore store: per sector its energies by eigenvector column, the
    kept column count (kept columns come first: a sector keeps its lowest states) and
    the eigenvector block."""
    nVar = st.nVar
    R = get_restore(st, N)
    si, bo, E = R["subspaceInfo"], R["basis_output"], R["eigenvalue"]
    nsub = si.shape[0]
    dims = si[:, nVar].astype(np.int64)
    Ecol = [np.zeros(int(d)) for d in dims]
    kept = np.zeros(nsub, dtype=np.int64)
    last = N == st.nIter
    for i in range(R["numberOfBasis_full"]):
        s = _find_subspace(si, nVar, bo[i, :nVar])
        c = int(bo[i, nVar]) - 1
        Ecol[s][c] = E[i]
        if i < R["numberOfBasis"] and not last:
            kept[s] += 1
    for s in range(nsub):
        assert np.all(np.diff(Ecol[s]) >= -1e-12)
    V = [R["eigenvector"][int(si[s, nVar + 1]) - 1:int(si[s, nVar + 1]) - 1 + int(dims[s]) ** 2]
         .reshape((int(dims[s]), int(dims[s])), order="F") for s in range(nsub)]
    return dict(R=R, si=si, dims=dims, Ecol=Ecol, kept=kept, V=V)


def fdm_weights(st: State, T: float, shells: Dict[int, dict]) -> Tuple[Dict[int, list], float]:
    """Boltzmann weight of every discarded state in the full density matrix,
    P_s = d^(N_max - N) exp(-eps_s / T) / Z, with eps_s = scale(N) E_s + C_N the energy
    on one scale for all shells (C_N = C_(N-1) + scale(N) min(H_N), the shifts the
    iterations subtract) and d = local states per site.  Returns P[N][sector] (per
    discarded column, kept columns 0) and ln Z."""
    N0, Nmax = st.startTrancation, st.nIter
    # C_N measured from C_Nmax: C_N - C_Nmax = -sum_(N' > N) scale(N') min(H_N'), small
    # numbers, so that eps / T keeps its precision at low T
    Cs = {Nmax: 0.0}
    for N in range(Nmax - 1, st.first - 1, -1):
        Cs[N] = Cs[N + 1] - st.scale(N + 1) * st.emin[N + 1]
    logs = []
    for N in range(N0, Nmax + 1):
        sh = shells[N]
        for s, Ec in enumerate(sh["Ecol"]):
            k = int(sh["kept"][s])
            eps = st.scale(N) * Ec[k:] + Cs[N]
            logs.append((Nmax - N) * math.log(st.nOps) - eps / T)
    allv = np.concatenate(logs) if logs else np.zeros(0)
    lmax = float(np.max(allv))
    lnZ = lmax + math.log(float(np.sum(np.exp(allv - lmax))))
    P: Dict[int, list] = {}
    for N in range(N0, Nmax + 1):
        sh = shells[N]
        P[N] = []
        for s, Ec in enumerate(sh["Ecol"]):
            k = int(sh["kept"][s])
            p = np.zeros(len(Ec))
            eps = st.scale(N) * Ec[k:] + Cs[N]
            p[k:] = np.exp((Nmax - N) * math.log(st.nOps) - eps / T - lnZ)
            P[N].append(p)
    return P, lnZ


def fdm_density(st: State, shells: Dict[int, dict], P: Dict[int, list]) -> Dict[int, list]:
    """Kept-space reduced density matrices R_N (per kept sector, columns in eigenvector
    order) by the backward recursion of reducedDensityMatrixDGEMM.F90:164-297, each
    child sector carrying its kept block R_(N+1) and the weights P of its discarded
    columns: R_S(N) = sum_op A_op blockdiag(R_child, diag(P_child)) A_op^T."""
    nVar, nOps = st.nVar, st.nOps
    N0, Nmax = st.startTrancation, st.nIter
    R: Dict[int, list] = {}
    for N in range(Nmax - 1, N0 - 1, -1):
        sh, ch = shells[N], shells[N + 1]
        csi, cbi = ch["si"], ch["R"]["basis_input"]
        R[N] = []
        for S in range(len(sh["dims"])):
            n = int(sh["kept"][S])
            rho = np.zeros((n, n))
            if n == 0:
                R[N].append(rho)
                continue
            qS = sh["si"][S, :nVar].astype(np.int64)
            for op in range(nOps):
                c = _find_subspace(csi, nVar, qS - st.operation[op, :nVar])
                if c is None:
                    continue
                dc = int(ch["dims"][c])
                b0 = int(csi[c, nVar + 2]) - 1
                var = cbi[b0:b0 + dc, nVar + 1]
                opr = cbi[b0:b0 + dc, nVar + 2] - 1
                A = np.zeros((n, dc))
                for il in range(n):
                    hit = np.nonzero((var == il + 1) & (opr == op))[0]
                    if len(hit):
                        A[il, :] = ch["V"][c][int(hit[0]), :]
                kc = int(ch["kept"][c])
                Dm = np.diag(P[N + 1][c])
                if kc > 0:
                    Dm[:kc, :kc] = R[N + 1][c]
                rho += A @ Dm @ A.T
            R[N].append(rho)
    return R


def fdm_spectrum(st: State, T: float):
    """FDM bins at temperature T (same grid and two-bin split as the CFS bins).  Per
    shell N and matrix type m, for each sector x and y = x + positive operation of m,
    M = <y|d^dag|x> (spectrumElementDGEMM) over all columns; the pairs not both kept
    contribute rho_x M^2 (particle added to x) and rho_y M^2 (particle taken from y) at
    omega = scale(N) (E_y - E_x), in the bins of the sign of omega, rho = P on discarded
    states and the matrix R on kept ones (the kept-discarded terms with R are the CFS
    terms).  Returns (binPos, binNeg, diagnostics)."""
    nVar = st.nVar
    N0, Nmax = st.startTrancation, st.nIter
    shells = {N: _shell(st, N) for N in range(N0, Nmax + 1)}
    P, lnZ = fdm_weights(st, T, shells)
    Rk = fdm_density(st, shells, P)
    # at every shell, the kept-space trace plus the weight of the states discarded up to
    # and including it is the whole trace, 1
    traces = {}
    done = 0.0
    for N in range(N0, Nmax + 1):
        done += sum(float(np.sum(p)) for p in P[N])
        traces[N] = done + (sum(float(np.trace(r)) for r in Rk[N]) if N < Nmax else 0.0)
    nbin = st.numberOfBin
    binPos = np.zeros((nbin * st.nMat, 2), order="F")
    binNeg = np.zeros((nbin * st.nMat, 2), order="F")
    binPos[:, 0] = st.binPos[:, 0]
    binNeg[:, 0] = st.binNeg[:, 0]
    for N in range(N0, Nmax + 1):
        sh = shells[N]
        si, R = sh["si"], sh["R"]
        sc = st.scale(N)
        for x in range(len(sh["dims"])):
            qx = si[x, :nVar].astype(np.int64)
            for m in range(st.nMat):
                y = _find_subspace(si, nVar, qx + st.pos_op[m])
                if y is None:
                    continue
                dx, dy = int(sh["dims"][x]), int(sh["dims"][y])
                M = spectrum_element_dgemm(st, R, y, dy, 0, x, dx, 0, m)      # (dy, dx)
                kx, ky = int(sh["kept"][x]), int(sh["kept"][y])
                Ex, Ey = sh["Ecol"][x], sh["Ecol"][y]
                w = (Ey[:, None] - Ex[None, :]) * sc                            # omega
                en = np.abs(w)
                M2 = M * M
                notkk = np.ones((dy, dx), dtype=bool)
                notkk[:ky, :kx] = False
                # rho_x: P on discarded columns of x; R_x on kept columns (rows y discarded)
                wpos = M2 * P[N][x][None, :]
                if kx > 0:
                    wpos[ky:, :kx] = M[ky:, :kx] * (M[ky:, :kx] @ Rk[N][x])
                wneg = M2 * P[N][y][:, None]
                if ky > 0:
                    wneg[:ky, kx:] = M[:ky, kx:] * (Rk[N][y] @ M[:ky, kx:])
                # both terms sit at omega = E_y - E_x: negative frequencies go to the
                # negative bins (at omega = 0 the x term to the positive, the y term to
                # the negative ones, as the T = 0 routines bin them)
                xpos = (w >= 0.0) & notkk
                ypos = (w > 0.0) & notkk
                xneg = (w < 0.0) & notkk
                yneg = (w <= 0.0) & notkk
                bin_spikes(st, binPos, np.concatenate([en[xpos], en[ypos]]),
                           np.concatenate([wpos[xpos], wneg[ypos]]), m)
                bin_spikes(st, binNeg, np.concatenate([en[xneg], en[yneg]]),
                           np.concatenate([wpos[xneg], wneg[yneg]]), m)
    return binPos, binNeg, dict(lnZ=lnZ, traces=traces)


def spectrum_lines(st: State):
    """The (energy, weight) rows main.F90:228-252 would write, per matrix type."""
    out = {}
    nbin = st.numberOfBin
    thr = 1.0e-16 * st.scale(st.nIter)
    for m in range(st.nMat):
        for name, cont in (("positive", st.binPos), ("negative", st.binNeg)):
            blk = cont[m * nbin:(m + 1) * nbin]
            sel = np.abs(blk[:, 1]) > thr
            out[(name, m + 1)] = blk[sel].copy()
    return out
