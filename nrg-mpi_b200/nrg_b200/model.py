"""Input side of the NRG hot path: model generators and the reference's input files.

The reference reads three files (reference files cited inline):

* ``parameter.txt``      namelist ``&nrg``             (module.F90:656-688)
* ``hamiltonianInfo.dat`` namelist ``&hamiltonianInfo`` (module.F90:846-862)
* ``initial.dat``        impurity eigenbasis, operator matrices, coefficient tables,
                         local operations and Wilson chain (read_initial_basis.F90:27-204)

``initial.dat`` is produced in the reference's world by an external Java program that is
not part of the reference.  This module is the replacement generator: it builds the
single-impurity Anderson model (SIAM) and the two-orbital Anderson model with Hund
coupling in the reference's conventions and writes the three files.  ``read_inputs``
reads them back exactly the way ``read_initial_basis.F90`` does, including the Wilson
chain rescale of ``read_initial_basis.F90:103-142``.

Conventions used by the generated tables (they are the reference's, derived from how
``diagonalization.F90``, ``invariantMatrixDGEMM.F90`` and
``invariantMatrixForSpectrumDGEMM.F90`` consume them):

* quantum numbers are ``(Q, 2Sz)`` with ``Q = n - (number of sites)`` (charge measured
  from half filling);
* a new product state is ``|r, j> = F_j^dagger |r>``: the local creation operators of
  the added site stand to the left of every operator of the old block, so
  ``basis_input%basis = basis_output%basis - operation(j, 1:nVar)``
  (prepareBasis.F90:47-48) with ``operation(j, 1:nVar) = -(Q_j, 2Sz_j)``;
* ``operation(j, nVar+c)`` is the occupation of chain ``c`` in local state ``j``
  (used as the on-site term, diagonalization.F90:166-171);
* ``invariant_matrix(r, l, t) = <l| f^dagger_t |r>`` (invariantMatrixDGEMM.F90:330);
* ``invariant_matrix_spectrum(r, l, m) = <l| d^dagger_m |r>``.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import Callable, Dict, List, Optional, Tuple

import numpy as np


# --------------------------------------------------------------------------------------
# data model
# --------------------------------------------------------------------------------------
@dataclasses.dataclass
class NrgInput:
    """Everything ``setupHamiltonian`` + ``read_parameter`` + ``read_initial_basis`` fill.

    Integer tables keep the reference's 1-based values.  Real matrices are Fortran
    column-major (``order='F'``) so that their flat memory matches the Fortran arrays.
    Chains are stored *raw* (as written to ``initial.dat``); ``rescaled_chains`` applies
    read_initial_basis.F90:103-142.
    """

    # &nrg (module.F90:612-626)
    bandWidth: float
    ztrick: float
    Lambda: float
    scalingType: int
    truncation: int
    # &hamiltonianInfo (module.F90:722-760)
    numberOfIteration: int
    numberOfChain: int
    numberOfVariation: int
    conservationBlock: np.ndarray  # int (2,2): row 1 charge (start,end), row 2 spin
    numberOfMatrix: int
    numberOfConductionMatrix: int
    numberOfBasis: int
    numberOfCoefficient: int
    numberOfOperation: int
    indexOfFirstIteration: int
    flag_spectrum: bool = True
    flag_BCS: bool = False
    numberOfBCSCoefficient: int = 0
    # initial.dat
    basis_output: np.ndarray = None          # int32 (nb, nVar+3)
    eigenvalue: np.ndarray = None            # f64 (nb,)
    invariant_matrix: np.ndarray = None      # f64 (nb, nb, nCM) F-order
    coefficient_invariant_matrix_type: np.ndarray = None  # int32 (nCoef, 3)
    coefficient_invariant_matrix: np.ndarray = None       # f64 (nCoef,)
    coefficient_diagonalization_type: np.ndarray = None   # int32 (nCoef, 4)
    coefficient_diagonalization: np.ndarray = None        # f64 (nCoef,)
    operation: np.ndarray = None             # int32 (nOps, nVar+nChain)
    chain_diagonal_raw: np.ndarray = None    # f64 (nIter+2, nChain), index 0..nIter+1
    chain_nondiagonal_raw: np.ndarray = None  # f64 (nIter+2-first, nChain), first..nIter+1
    coefficient_invariant_matrix_spectrum: np.ndarray = None  # f64 (nMat, nOps)
    invariant_matrix_spectrum: np.ndarray = None  # f64 (nb, nb, nMat) F-order
    conservation_difference_spectrum: np.ndarray = None  # int32 (nMat, nVar)
    positiveSpectrumOperation: np.ndarray = None   # int32 (nMat, nVar)
    negativeSpectrumOperation: np.ndarray = None   # int32 (nMat, nVar)
    chain_BCS_raw: Optional[np.ndarray] = None     # f64 (nIter+2, nChain)
    coefficient_BCS: Optional[np.ndarray] = None   # int32 (nBCS, 3)
    description: str = ""

    # ---------------------------------------------------------------------------
    def scale(self, N: int) -> float:
        """Energy scale of iteration N (module.F90:690-711)."""
        L, z, D = self.Lambda, self.ztrick, self.bandWidth
        if self.scalingType == 0:
            return L ** (-float(N) * 0.5)
        if self.scalingType == 1:
            return D * 0.5 * (1.0 + 1.0 / L) * L ** (-float(N) * 0.5 - z + 1.0)
        if self.scalingType == 2:
            return L ** (-float(N) * 0.5 - z) * D * (L - 1.0) / math.log(L)
        raise ValueError("scalingType must be 0, 1 or 2")

    def rescaled_chains(self):
        """Chain rescale of read_initial_basis.F90:103-142.

        Returns ``(chain_diagonal, chain_nondiagonal, chain_BCS)`` with the same index
        ranges as the raw arrays.  As in the reference the rescale loop runs over
        ``ii = 0 .. numberOfIteration+1`` only, so ``chain_nondiagonal(-1)`` (the
        impurity hybridisation) is used as written in ``initial.dat``.
        """
        L, z, D = self.Lambda, self.ztrick, self.bandWidth
        first = self.indexOfFirstIteration
        cd = self.chain_diagonal_raw.copy()
        cn = self.chain_nondiagonal_raw.copy()
        for ii in range(0, self.numberOfIteration + 2):
            if self.scalingType == 0:
                fd = L ** (float(ii - 1) * 0.5)
                fn = L ** (float(ii) * 0.5)
            elif self.scalingType == 2:
                fd = L ** (float(ii - 1) * 0.5 + z) * math.log(L) / D / (L - 1.0)
                fn = L ** (float(ii) * 0.5 + z) * math.log(L) / D / (L - 1.0)
            elif self.scalingType == 1:
                fd = L ** (float(ii - 1) * 0.5 + z - 1.0) / D * 2.0 / (1.0 + 1.0 / L)
                fn = L ** (float(ii) * 0.5 + z - 1.0) / D * 2.0 / (1.0 + 1.0 / L)
            else:
                raise ValueError("scalingType")
            cd[ii, :] = cd[ii, :] * fd
            cn[ii - first, :] = cn[ii - first, :] * fn
        return cd, cn, (None if self.chain_BCS_raw is None else self.chain_BCS_raw.copy())

    @property
    def nVar(self):
        return self.numberOfVariation


# --------------------------------------------------------------------------------------
# Wilson chain for a flat band (Wilson's logarithmic discretisation, z = 1)
# --------------------------------------------------------------------------------------
def wilson_flat_band_hoppings(Lambda: float, D: float, n_sites: int) -> np.ndarray:
    """Hopping t_n (n = 0..n_sites-1) of the Wilson chain for a flat band of half width D.

    Wilson, Rev. Mod. Phys. 47, 773 (1975), eq. (2.15):
    t_n = D (1+1/L)/2 * (1 - L^{-n-1}) L^{-n/2} / sqrt((1 - L^{-2n-1})(1 - L^{-2n-3})).
    The on-site energies vanish for the particle-hole symmetric flat band.
    """
    n = np.arange(n_sites, dtype=np.float64)
    L = float(Lambda)
    return (D * 0.5 * (1.0 + 1.0 / L) * (1.0 - L ** (-n - 1.0)) * L ** (-n / 2.0)
            / np.sqrt((1.0 - L ** (-2.0 * n - 1.0)) * (1.0 - L ** (-2.0 * n - 3.0))))


def _a_lambda(Lambda: float) -> float:
    """Wilson's discretisation correction A_Lambda = (1+1/L)/2 * ln L / (1-1/L)."""
    L = float(Lambda)
    return 0.5 * (1.0 + 1.0 / L) * math.log(L) / (1.0 - 1.0 / L)


# --------------------------------------------------------------------------------------
# local site algebra (one spinful orbital per chain)
# --------------------------------------------------------------------------------------
class _Fock:
    """Fock states of ``n_modes`` fermion modes as bit masks, creation order by mode index.

    A state with occupied modes m1 < m2 < ... is ``c^dag_{m1} c^dag_{m2} ... |0>``.
    """

    def __init__(self, n_modes: int):
        self.n = n_modes

    def apply_cdag(self, mode: int, state: int):
        if state >> mode & 1:
            return None, 0
        # sign: number of occupied modes with index < mode
        below = bin(state & ((1 << mode) - 1)).count("1")
        return state | (1 << mode), (-1) ** below

    def apply_c(self, mode: int, state: int):
        if not (state >> mode & 1):
            return None, 0
        below = bin(state & ((1 << mode) - 1)).count("1")
        return state & ~(1 << mode), (-1) ** below

    @staticmethod
    def count(state: int) -> int:
        return bin(state).count("1")


def _local_site_tables(n_chain: int):
    """Local states of one added Wilson site (``n_chain`` spinful chains) and tables.

    Modes: (chain c, spin s) -> mode 2c+s, s=0 up, s=1 down.  Returns
    ``(states, qn, occ, fdag)`` where ``fdag[t][(a, b)] = <a|f^dag_t|b>`` with
    ``t = 2c+s``.
    """
    n_modes = 2 * n_chain
    fock = _Fock(n_modes)
    states = list(range(1 << n_modes))
    # order: by total occupation, then by bit pattern (deterministic, documented)
    states.sort(key=lambda s: (fock.count(s), s))
    idx = {s: i for i, s in enumerate(states)}
    qn = []
    occ = []
    for s in states:
        n = fock.count(s)
        two_sz = sum(1 if (s >> m & 1) and m % 2 == 0 else 0 for m in range(n_modes)) - \
            sum(1 if (s >> m & 1) and m % 2 == 1 else 0 for m in range(n_modes))
        qn.append((n - n_chain, two_sz))
        occ.append([fock.count(s & (0b11 << (2 * c))) for c in range(n_chain)])
    fdag = []
    for t in range(n_modes):
        mat = {}
        for b in states:
            a, sg = fock.apply_cdag(t, b)
            if a is not None:
                mat[(idx[a], idx[b])] = float(sg)
        fdag.append(mat)
    return states, qn, occ, fdag


# --------------------------------------------------------------------------------------
# generic builder from an impurity Hamiltonian in a Fock basis
# --------------------------------------------------------------------------------------
def _build(imp_modes: int, h_imp: np.ndarray, n_chain: int, Lambda: float, D: float,
           hyb: List[float], n_iter: int, n_keep: int, description: str,
           with_spectrum: bool = True, a_lambda: bool = True,
           chain: Optional[Tuple[np.ndarray, np.ndarray]] = None) -> NrgInput:
    """Assemble an :class:`NrgInput` for an impurity with ``imp_modes`` fermion modes.

    ``h_imp`` is the impurity Hamiltonian in the Fock basis of ``imp_modes`` modes (bit
    masks, dense).  Impurity mode ``2c+s`` hybridises with Wilson chain ``c`` spin ``s``
    with strength ``hyb[c]`` (already the physical V).  The impurity block is
    diagonalised per (Q, 2Sz) sector; its eigenstates become the initial
    ``basis_output``.  ``chain = (eps, t)`` (physical units, at least numberOfIteration+2
    on-site energies and hoppings) replaces the flat band's Wilson chain in every chain.
    """
    scalingType, z = 1, 1.0
    first = -1
    nVar = 2
    nOps = 1 << (2 * n_chain)
    nCM = 2 * n_chain
    fock = _Fock(imp_modes)
    n_imp_sites = imp_modes // 2

    def scale(N):
        return D * 0.5 * (1.0 + 1.0 / Lambda) * Lambda ** (-float(N) * 0.5 - z + 1.0)

    # ---- impurity eigenbasis, sectors by (Q, 2Sz)
    dim = 1 << imp_modes
    qn_of = []
    for s in range(dim):
        n = fock.count(s)
        up = sum(1 for m in range(0, imp_modes, 2) if s >> m & 1)
        dn = sum(1 for m in range(1, imp_modes, 2) if s >> m & 1)
        qn_of.append((n - n_imp_sites, up - dn))
    sectors: Dict[tuple, list] = {}
    for s in range(dim):
        sectors.setdefault(qn_of[s], []).append(s)
    eig_states = []   # list of (qn, column index 1-based, energy, vector over fock states)
    for q in sorted(sectors):
        members = sectors[q]
        h = h_imp[np.ix_(members, members)]
        w, v = np.linalg.eigh(h)
        for c in range(len(members)):
            vec = np.zeros(dim)
            vec[members] = v[:, c]
            eig_states.append((q, c + 1, float(w[c]), vec))
    nb = len(eig_states)
    basis_output = np.zeros((nb, nVar + 3), dtype=np.int32)
    eigenvalue = np.zeros(nb)
    V = np.zeros((dim, nb))
    for i, (q, c, e, vec) in enumerate(eig_states):
        basis_output[i, 0:2] = q
        basis_output[i, 2] = c
        eigenvalue[i] = e / scale(first - 1)   # "eigenvalue is scaled already"
        V[:, i] = vec

    # ---- operator matrices <l| op |r> in the eigenbasis
    def opmat(mode):
        M = np.zeros((dim, dim))
        for b in range(dim):
            a, sg = fock.apply_cdag(mode, b)
            if a is not None:
                M[a, b] = sg
        return V.T @ M @ V   # (l, r) = <l|c^dag|r>

    # conduction-type matrices: impurity mode of chain c couples to chain c, t = 2c+s
    im = np.zeros((nb, nb, nCM), order="F")
    for t in range(nCM):
        im[:, :, t] = opmat(t).T   # invariant_matrix(r, l, t) = <l|d^dag_t|r>
    im[np.abs(im) < 1e-15] = 0.0

    # ---- local site tables
    states, lqn, locc, fdag = _local_site_tables(n_chain)
    operation = np.zeros((nOps, nVar + n_chain), dtype=np.int32)
    for j in range(nOps):
        operation[j, 0] = -lqn[j][0]
        operation[j, 1] = -lqn[j][1]
        operation[j, 2:2 + n_chain] = locc[j]
    nl = [sum(o) for o in locc]
    # diagonalisation coefficients: <r_i, a| f^dag_N f_{N+1} |r_j, b> = (-1)^{n_a}<a|f|b>
    # entry (a, b, type, channel, coef) for b = f^dag_t a
    diag_rows = []
    im_rows = []
    for t in range(nCM):
        for (a_, b_), v in sorted(fdag[t].items(), key=lambda kv: (kv[0][1], kv[0][0])):
            # fdag[t][(a, b)] = <a|f^dag_t|b>, a has one more electron
            # hopping row: (lower, upper) = (b_, a_)
            diag_rows.append((b_ + 1, a_ + 1, t + 1, t // 2 + 1, ((-1) ** nl[b_]) * v))
            # invariant matrix of the new site: <left|f^dag_t|right> with left = a_
            im_rows.append((a_ + 1, b_ + 1, t + 1, v))
    nCoef = len(diag_rows)
    assert len(im_rows) == nCoef
    cdt = np.array([r[:4] for r in diag_rows], dtype=np.int32)
    cd = np.array([r[4] for r in diag_rows], dtype=np.float64)
    cit = np.array([r[:3] for r in im_rows], dtype=np.int32)
    ci = np.array([r[3] for r in im_rows], dtype=np.float64)

    # ---- Wilson chain (physical units, as in initial.dat; rescaled by the reader)
    n_pts = n_iter + 2
    t_n = wilson_flat_band_hoppings(Lambda, D, n_pts) if chain is None else np.asarray(chain[1][:n_pts])
    e_n = np.zeros(n_pts) if chain is None else np.asarray(chain[0][:n_pts])
    if len(t_n) != n_pts or len(e_n) != n_pts:
        raise ValueError(f"the chain needs {n_pts} on-site energies and hoppings")
    chain_diag = np.zeros((n_pts, n_chain))
    chain_nond = np.zeros((n_pts - first, n_chain))
    for c in range(n_chain):
        chain_diag[:, c] = e_n           # site n's energy, added at iteration n-1
        chain_nond[1:, c] = t_n          # indices 0..n_iter+1
        chain_nond[0, c] = hyb[c] / scale(first)   # index -1: used as written

    inp = NrgInput(
        bandWidth=D, ztrick=z, Lambda=Lambda, scalingType=scalingType, truncation=n_keep,
        numberOfIteration=n_iter, numberOfChain=n_chain, numberOfVariation=nVar,
        conservationBlock=np.array([[1, 1], [2, 2]], dtype=np.int32),
        numberOfMatrix=nCM if with_spectrum else 0, numberOfConductionMatrix=nCM,
        numberOfBasis=nb, numberOfCoefficient=nCoef, numberOfOperation=nOps,
        indexOfFirstIteration=first, flag_spectrum=with_spectrum,
        basis_output=basis_output, eigenvalue=eigenvalue, invariant_matrix=im,
        coefficient_invariant_matrix_type=cit, coefficient_invariant_matrix=ci,
        coefficient_diagonalization_type=cdt, coefficient_diagonalization=cd,
        operation=operation, chain_diagonal_raw=chain_diag, chain_nondiagonal_raw=chain_nond,
        description=description,
    )
    if with_spectrum:
        nMat = nCM
        sign = np.array([(-1.0) ** n for n in nl])
        inp.coefficient_invariant_matrix_spectrum = np.tile(sign, (nMat, 1))
        inp.invariant_matrix_spectrum = np.asfortranarray(im.copy())
        cds = np.zeros((nMat, nVar), dtype=np.int32)
        for m in range(nMat):
            cds[m] = (1, 1 if m % 2 == 0 else -1)
        inp.conservation_difference_spectrum = cds
        inp.positiveSpectrumOperation = cds.copy()
        inp.negativeSpectrumOperation = -cds
    return inp


def siam(U: float, Gamma: float, eps_d: Optional[float] = None, Lambda: float = 2.5,
         n_keep: int = 512, n_iterations: int = 40, D: float = 1.0,
         a_lambda: bool = True) -> NrgInput:
    """Single-impurity Anderson model, flat band, one Wilson chain, U(1)_Q x U(1)_Sz.

    ``n_iterations`` counts the calls of ``nrgIteration`` (main.F90:175-177): the loop
    runs over ``indexOfFirstIteration=-1 .. numberOfIteration`` so
    ``numberOfIteration = n_iterations - 2``.
    """
    if eps_d is None:
        eps_d = -U / 2.0
    h = np.zeros((4, 4))
    # modes: 0 = up, 1 = down; states as bit masks
    for s in range(4):
        n_up, n_dn = s & 1, (s >> 1) & 1
        h[s, s] = eps_d * (n_up + n_dn) + U * n_up * n_dn
    g_eff = Gamma * (_a_lambda(Lambda) if a_lambda else 1.0)
    V = math.sqrt(2.0 * D * g_eff / math.pi)
    desc = (f"SIAM U={U} Gamma={Gamma} eps_d={eps_d} Lambda={Lambda} N_keep={n_keep} "
            f"iterations={n_iterations}")
    return _build(2, h, 1, Lambda, D, [V], n_iterations - 2, n_keep, desc,
                  a_lambda=a_lambda)


def siam_bath(U: float, eps_d: float, hybridization: Callable[[float], float], Lambda: float = 2.0,
              n_keep: int = 512, n_iterations: int = 40, D: float = 1.0, scheme: str = "campo",
              name: str = "") -> NrgInput:
    """Single-impurity Anderson model with an arbitrary bath: ``hybridization(eps)`` is
    Gamma(eps) = pi sum_k |V_k|^2 delta(eps - eps_k) on [-D, D] (energies in the units of
    D).  The Wilson chain (on-site energies and hoppings) comes from its logarithmic
    discretisation with the ``scheme``'s representative energies ("campo": Campo and
    Oliveira, no A_Lambda correction; "wilson": interval means, as for siam() without
    a_lambda), z = 1; see nrg_b200.chain."""
    from . import chain as _chain
    n_pts = n_iterations                      # numberOfIteration + 2 chain sites used
    V, e, t = _chain.log_discretized_chain(hybridization, D, Lambda, n_pts + 1, 1.0, scheme)
    h = np.zeros((4, 4))
    for st in range(4):
        n_up, n_dn = st & 1, (st >> 1) & 1
        h[st, st] = eps_d * (n_up + n_dn) + U * n_up * n_dn
    desc = (f"SIAM bath {name or 'custom'} ({scheme}) U={U} eps_d={eps_d} Lambda={Lambda} "
            f"N_keep={n_keep} iterations={n_iterations}")
    return _build(2, h, 1, Lambda, D, [V], n_iterations - 2, n_keep, desc, a_lambda=False,
                  chain=(e, t))


def two_orbital_hund(U: float = 0.2, J: float = 0.02, Gamma: float = 0.015,
                     eps_d: Optional[float] = None, Lambda: float = 3.0,
                     n_keep: int = 8192, n_iterations: int = 40, D: float = 1.0) -> NrgInput:
    """Two-orbital Anderson model with Hund coupling, two Wilson chains (16 local states).

    H_imp = eps_d N + U sum_a n_a,up n_a,dn + (U - 2J) sum_{a<b} n_a n_b ... in the
    density-density Kanamori form with Hund exchange -J (S_1 . S_2) omitted beyond its
    Ising part (kept U(1)_Q x U(1)_Sz).  eps_d defaults to the particle-hole symmetric
    value -(3U - 5J)/2.
    """
    U2 = U - 2.0 * J
    U3 = U - 3.0 * J
    if eps_d is None:
        eps_d = -(U + U2 + U3) / 2.0
    dim = 16
    h = np.zeros((dim, dim))
    for s in range(dim):
        n = [(s >> m) & 1 for m in range(4)]  # modes: orb a spin s -> 2a+s
        N = sum(n)
        e = eps_d * N
        e += U * (n[0] * n[1] + n[2] * n[3])
        e += U2 * (n[0] * n[3] + n[1] * n[2])   # opposite spins, different orbitals
        e += U3 * (n[0] * n[2] + n[1] * n[3])   # same spin, different orbitals
        h[s, s] = e
    g_eff = Gamma * _a_lambda(Lambda)
    V = math.sqrt(2.0 * D * g_eff / math.pi)
    desc = (f"2-orbital Hund U={U} J={J} Gamma={Gamma} Lambda={Lambda} N_keep={n_keep} "
            f"iterations={n_iterations}")
    return _build(4, h, 2, Lambda, D, [V, V], n_iterations - 2, n_keep, desc)


# --------------------------------------------------------------------------------------
# the reference's input files
# --------------------------------------------------------------------------------------
def _fbool(b: bool) -> str:
    return ".true." if b else ".false."


def write_inputs(inp: NrgInput, directory: str) -> None:
    """Write parameter.txt, hamiltonianInfo.dat and initial.dat in the reference's formats."""
    os.makedirs(directory, exist_ok=True)
    with open(os.path.join(directory, "parameter.txt"), "w") as f:
        f.write("&nrg\n")
        f.write(f" bandWidth = {float(inp.bandWidth)!r}, ztrick = {float(inp.ztrick)!r}, "
                f"Lambda = {float(inp.Lambda)!r}, scalingType = {inp.scalingType},\n")
        f.write(f" truncation = {inp.truncation}, cfsnrg = .false., noimpurity = .false.,\n")
        f.write(" loadRestart = .false., saveRestart = .false.\n/\n")
    cb = inp.conservationBlock
    with open(os.path.join(directory, "hamiltonianInfo.dat"), "w") as f:
        f.write("&hamiltonianInfo\n")
        f.write(f" numberOfIteration = {inp.numberOfIteration}, numberOfChain = {inp.numberOfChain},\n")
        f.write(f" numberOfVariation = {inp.numberOfVariation},\n")
        # column-major namelist order: (1,1) (2,1) (1,2) (2,2)
        f.write(f" conservationBlock = {cb[0,0]}, {cb[1,0]}, {cb[0,1]}, {cb[1,1]},\n")
        f.write(f" numberOfMatrix = {inp.numberOfMatrix}, "
                f"numberOfConductionMatrix = {inp.numberOfConductionMatrix},\n")
        f.write(f" numberOfBasis = {inp.numberOfBasis}, numberOfCoefficient = {inp.numberOfCoefficient},\n")
        f.write(f" numberOfBCSCoefficient = {inp.numberOfBCSCoefficient}, numberOfCoefficientImpurity = 0,\n")
        f.write(f" numberOfOperation = {inp.numberOfOperation}, "
                f"indexOfFirstIteration = {inp.indexOfFirstIteration},\n")
        f.write(f" flag_spectrum = {_fbool(inp.flag_spectrum)}, flag_local = .false., "
                f"flag_BCS = {_fbool(inp.flag_BCS)}\n/\n")
    nb, nVar = inp.numberOfBasis, inp.numberOfVariation
    lines = []
    w = lines.append
    w("basis")
    for i in range(nb):
        w(" ".join(str(int(x)) for x in inp.basis_output[i, :nVar + 1]) + f" {float(inp.eigenvalue[i])!r}")
    w("invariant_matrix")
    for t in range(inp.numberOfConductionMatrix):
        for j in range(nb):
            for k in range(nb):
                w(repr(float(inp.invariant_matrix[k, j, t])))
    w("coefficient_invariant_matrix")
    for i in range(inp.numberOfCoefficient):
        r = inp.coefficient_invariant_matrix_type[i]
        w(f"{r[0]} {r[1]} {r[2]} {float(inp.coefficient_invariant_matrix[i])!r}")
    w("coefficient_diagonalization")
    for i in range(inp.numberOfCoefficient):
        r = inp.coefficient_diagonalization_type[i]
        w(f"{r[0]} {r[1]} {r[2]} {r[3]} {float(inp.coefficient_diagonalization[i])!r}")
    w("operation")
    for i in range(inp.numberOfOperation):
        w(" ".join(str(int(x)) for x in inp.operation[i]))
    w("chain")
    first = inp.indexOfFirstIteration
    for c in range(inp.numberOfChain):
        w(f"chain_diagonal_{c+1}")
        for j in range(0, inp.numberOfIteration + 2):
            w(repr(float(inp.chain_diagonal_raw[j, c])))
    for c in range(inp.numberOfChain):
        w(f"chain_nondiagonal_{c+1}")
        for j in range(first, inp.numberOfIteration + 2):
            w(repr(float(inp.chain_nondiagonal_raw[j - first, c])))
    if inp.flag_spectrum:
        w("coefficient_invariant_matrix_spectrum")
        for m in range(inp.numberOfMatrix):
            for i in range(inp.numberOfOperation):
                w(repr(float(inp.coefficient_invariant_matrix_spectrum[m, i])))
        w("invariant_matrix_spectrum")
        for m in range(inp.numberOfMatrix):
            for j in range(nb):
                for i in range(nb):
                    w(repr(float(inp.invariant_matrix_spectrum[i, j, m])))
        w("conservation_difference_spectrum")
        for m in range(inp.numberOfMatrix):
            w(" ".join(str(int(x)) for x in inp.conservation_difference_spectrum[m]))
        w("positiveSpectrumOperation")
        for m in range(inp.numberOfMatrix):
            w(" ".join(str(int(x)) for x in inp.positiveSpectrumOperation[m]))
        w("negativeSpectrumOperation")
        for m in range(inp.numberOfMatrix):
            w(" ".join(str(int(x)) for x in inp.negativeSpectrumOperation[m]))
    if inp.flag_BCS:
        for c in range(inp.numberOfChain):
            w(f"chain_BCS_{c+1}")
            for j in range(0, inp.numberOfIteration + 2):
                w(repr(float(inp.chain_BCS_raw[j, c])))
        w("coefficient_BCS")
        for i in range(inp.numberOfBCSCoefficient):
            w(" ".join(str(int(x)) for x in inp.coefficient_BCS[i]))
    with open(os.path.join(directory, "initial.dat"), "w") as f:
        f.write("\n".join(lines) + "\n")


def _parse_namelist(path: str) -> Dict[str, str]:
    txt = open(path).read()
    start = txt.index("&")
    body = txt[start:]
    body = body[body.index("\n"):] if "\n" in body else body
    body = body.rsplit("/", 1)[0]
    out: Dict[str, List[str]] = {}
    key = None
    for tok in body.replace("\n", " ").split(","):
        tok = tok.strip()
        if not tok:
            continue
        if "=" in tok:
            k, v = tok.split("=", 1)
            key = k.strip()
            out[key] = [v.strip()]
        elif key is not None:
            out[key].append(tok)
    return {k: ",".join(v) for k, v in out.items()}


def _fval(s: str) -> float:
    return float(s.lower().replace("d", "e"))


def _lval(s: str) -> bool:
    return s.strip().lower().strip(".").startswith("t")


def read_inputs(directory: str) -> NrgInput:
    """Read the three input files (module.F90:656-688, 846-880; read_initial_basis.F90)."""
    p = _parse_namelist(os.path.join(directory, "parameter.txt"))
    h = _parse_namelist(os.path.join(directory, "hamiltonianInfo.dat"))
    cbf = [int(x) for x in h["conservationBlock"].split(",")]
    cb = np.array([[cbf[0], cbf[2]], [cbf[1], cbf[3]]], dtype=np.int32)
    inp = NrgInput(
        bandWidth=_fval(p["bandWidth"]), ztrick=_fval(p["ztrick"]), Lambda=_fval(p["Lambda"]),
        scalingType=int(p["scalingType"]), truncation=int(p["truncation"]),
        numberOfIteration=int(h["numberOfIteration"]), numberOfChain=int(h["numberOfChain"]),
        numberOfVariation=int(h["numberOfVariation"]), conservationBlock=cb,
        numberOfMatrix=int(h["numberOfMatrix"]),
        numberOfConductionMatrix=int(h["numberOfConductionMatrix"]),
        numberOfBasis=int(h["numberOfBasis"]), numberOfCoefficient=int(h["numberOfCoefficient"]),
        numberOfOperation=int(h["numberOfOperation"]),
        indexOfFirstIteration=int(h["indexOfFirstIteration"]),
        flag_spectrum=_lval(h.get("flag_spectrum", ".false.")),
        flag_BCS=_lval(h.get("flag_BCS", ".false.")),
        numberOfBCSCoefficient=int(h.get("numberOfBCSCoefficient", "0")),
    )
    nb, nVar, nCM = inp.numberOfBasis, inp.numberOfVariation, inp.numberOfConductionMatrix
    with open(os.path.join(directory, "initial.dat")) as f:
        lines = [ln.split() for ln in f.read().splitlines() if ln.strip()]
    pos = 0

    def nxt():
        nonlocal pos
        r = lines[pos]
        pos += 1
        return r

    nxt()
    inp.basis_output = np.zeros((nb, nVar + 3), dtype=np.int32)
    inp.eigenvalue = np.zeros(nb)
    for i in range(nb):
        r = nxt()
        inp.basis_output[i, :nVar + 1] = [int(x) for x in r[:nVar + 1]]
        inp.eigenvalue[i] = _fval(r[nVar + 1])
    nxt()
    im = np.zeros((nb, nb, nCM), order="F")
    for t in range(nCM):
        for j in range(nb):
            for k in range(nb):
                im[k, j, t] = _fval(nxt()[0])
    inp.invariant_matrix = im
    nxt()
    nC = inp.numberOfCoefficient
    inp.coefficient_invariant_matrix_type = np.zeros((nC, 3), dtype=np.int32)
    inp.coefficient_invariant_matrix = np.zeros(nC)
    for i in range(nC):
        r = nxt()
        inp.coefficient_invariant_matrix_type[i] = [int(x) for x in r[:3]]
        inp.coefficient_invariant_matrix[i] = _fval(r[3])
    nxt()
    inp.coefficient_diagonalization_type = np.zeros((nC, 4), dtype=np.int32)
    inp.coefficient_diagonalization = np.zeros(nC)
    for i in range(nC):
        r = nxt()
        inp.coefficient_diagonalization_type[i] = [int(x) for x in r[:4]]
        inp.coefficient_diagonalization[i] = _fval(r[4])
    nxt()
    nOps, nChain = inp.numberOfOperation, inp.numberOfChain
    inp.operation = np.zeros((nOps, nVar + nChain), dtype=np.int32)
    for i in range(nOps):
        inp.operation[i] = [int(x) for x in nxt()[:nVar + nChain]]
    nxt()
    first, nIter = inp.indexOfFirstIteration, inp.numberOfIteration
    inp.chain_diagonal_raw = np.zeros((nIter + 2, nChain))
    inp.chain_nondiagonal_raw = np.zeros((nIter + 2 - first, nChain))
    for c in range(nChain):
        nxt()
        for j in range(0, nIter + 2):
            inp.chain_diagonal_raw[j, c] = _fval(nxt()[0])
    for c in range(nChain):
        nxt()
        for j in range(first, nIter + 2):
            inp.chain_nondiagonal_raw[j - first, c] = _fval(nxt()[0])
    if inp.flag_spectrum:
        nMat = inp.numberOfMatrix
        nxt()
        inp.coefficient_invariant_matrix_spectrum = np.zeros((nMat, nOps))
        for m in range(nMat):
            for i in range(nOps):
                inp.coefficient_invariant_matrix_spectrum[m, i] = _fval(nxt()[0])
        nxt()
        ims = np.zeros((nb, nb, nMat), order="F")
        for m in range(nMat):
            for j in range(nb):
                for i in range(nb):
                    ims[i, j, m] = _fval(nxt()[0])
        inp.invariant_matrix_spectrum = ims
        for attr in ("conservation_difference_spectrum", "positiveSpectrumOperation",
                     "negativeSpectrumOperation"):
            nxt()
            arr = np.zeros((nMat, nVar), dtype=np.int32)
            for m in range(nMat):
                arr[m] = [int(x) for x in nxt()[:nVar]]
            setattr(inp, attr, arr)
    if inp.flag_BCS:
        inp.chain_BCS_raw = np.zeros((nIter + 2, nChain))
        for c in range(nChain):
            nxt()
            for j in range(0, nIter + 2):
                inp.chain_BCS_raw[j, c] = _fval(nxt()[0])
        nxt()
        nB = inp.numberOfBCSCoefficient
        inp.coefficient_BCS = np.zeros((nB, 3), dtype=np.int32)
        for i in range(nB):
            inp.coefficient_BCS[i] = [int(x) for x in nxt()[:3]]
    return inp


# --------------------------------------------------------------------------------------
# the five named workloads
# --------------------------------------------------------------------------------------
def config(n: int, **overrides) -> NrgInput:
    """The synthetic workloads, numbered as in the project's benchmark table.

    1: SIAM L=2.5 U=0.1 G=0.01 eps=-U/2, N_keep=512, 40 iterations (CPU-runnable)
    2: SIAM L=2.0 U=0.2 G=0.02 eps=-0.1, N_keep=2048, 60 iterations (plain FP64 bench)
    3: SIAM L=2.0 U=0.3 G=0.03 eps=-0.15, N_keep=4096, 60 iterations
    4: two-orbital Hund U=0.2 J=0.02 G=0.015, L=3, N_keep=8192, 40 iterations
    """
    if n == 1:
        kw = dict(U=0.1, Gamma=0.01, eps_d=-0.05, Lambda=2.5, n_keep=512, n_iterations=40)
        kw.update(overrides)
        return siam(**kw)
    if n == 2:
        kw = dict(U=0.2, Gamma=0.02, eps_d=-0.1, Lambda=2.0, n_keep=2048, n_iterations=60)
        kw.update(overrides)
        return siam(**kw)
    if n == 3:
        kw = dict(U=0.3, Gamma=0.03, eps_d=-0.15, Lambda=2.0, n_keep=4096, n_iterations=60)
        kw.update(overrides)
        return siam(**kw)
    if n == 4:
        kw = dict(U=0.2, J=0.02, Gamma=0.015, Lambda=3.0, n_keep=8192, n_iterations=40)
        kw.update(overrides)
        return two_orbital_hund(**kw)
    raise ValueError("config must be 1..4")
