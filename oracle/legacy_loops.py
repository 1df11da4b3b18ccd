"""Second oracle: the reference's loop-form routines, restated element by element.

TEST INFRASTRUCTURE, like ``nrg_oracle.py``: only ``tests/`` import it.

The reference keeps, beside the DGEMM routines it links, the older loop-form versions of
the same contractions (not in the Makefile's objects, or their call commented out):
invariantMatrix.F90, invariantMatrixForSpectrum.F90, reducedDensityMatrix.F90 and
calculateSpectrum.F90 with ``spectrumElement`` (module.F90:1127-1207).  They compute every
matrix element as an explicit sum over basis states, indexing the eigenvector blocks as
``eigenvector(count_eigenvector + dimension*(column-1) + (row-1))``, i.e. column-major
columns.  The DGEMM oracle reads the slice typo of the DGEMM routines
(invariantMatrixDGEMM.F90:223,227) with the same column semantics; these loops pin that
reading and the other index conventions independently of the GEMM formulation.

Each function takes the oracle's ``State`` at the point where the reference would call the
routine and returns the result instead of storing it, so that a test can compare it with
the DGEMM oracle's.  Pure Python loops: small cases only.

Differences between the two forms, restated as they are:
* invariantMatrix: one matrix type per (operation_left, operation_right) pair, the last
  matching coefficient row (invariantMatrix.F90:171-178); the DGEMM form fills every type
  that has a matching row.  They agree when each pair has one type (true for the models
  here).
* spikeZeroTemperature: the loop form takes the ground state's own column (gsVariation,
  calculateSpectrum.F90:76,110-112), the DGEMM form always column 1
  (calculateSpectrumDGEMM.F90:107-111).  They agree when no sector holds two ground states.
"""
from __future__ import annotations

from typing import Dict, List, Optional

import numpy as np

DEGENERACY_THRESHOLD = 1.0e-8      # module.F90:7


def _sector_of(si: np.ndarray, nVar: int, qn) -> Optional[int]:
    """The subspace loops of invariantMatrix.F90:131-145: the last sector whose quantum
    numbers match (the loop has no exit)."""
    hit = None
    for isub in range(si.shape[0]):
        if all(int(qn[v]) == int(si[isub, v]) for v in range(nVar)):
            hit = isub
    return hit


def invariant_matrix(st) -> np.ndarray:
    """invariantMatrix.F90:66-196 on one rank: <ileft| f^dagger_t |iright> for every pair
    of kept states, by sums over the basis states of the two sectors."""
    nVar, nb = st.nVar, st.nb
    si, bi, bo, V = st.subspaceInfo, st.basis_input, st.basis_output, st.eigenvector
    im = np.zeros((nb, nb, st.nCM), order="F")
    cs, ce = int(st.cb[0, 0]), int(st.cb[0, 1])       # conservationBlock (:73-76)
    ss, se = int(st.cb[1, 0]), int(st.cb[1, 1])
    ctype = st.cim_type                               # coefficient_invariant_matrix_type
    cval = st.cim                                     # coefficient_invariant_matrix
    sec = [_sector_of(si, nVar, bo[i, :nVar]) for i in range(nb)]
    # the coefficient scan (:171-178) depends only on the two operations: its outcome, the
    # last matching row, is tabulated once
    lookup = {}
    for op_a in range(1, st.nOps + 1):
        for op_b in range(1, st.nOps + 1):
            for icoef in range(ctype.shape[0]):
                if op_a == ctype[icoef, 0] and op_b == ctype[icoef, 1]:
                    lookup[(op_a, op_b)] = (float(cval[icoef]), int(ctype[icoef, 2]))
    for ileft in range(nb):
        ql = bo[ileft, :nVar].astype(np.int64)
        for iright in range(nb):
            qr = bo[iright, :nVar].astype(np.int64)
            dS = int(np.sum(ql[ss - 1:se] - qr[ss - 1:se]))
            if cs == ce and cs == 0:                           # :105-114
                if abs(dS) != 1:
                    continue
            else:                                              # :116-126
                dQ = int(np.sum(ql[cs - 1:ce] - qr[cs - 1:ce]))
                if dQ != 1 or abs(dS) != 1:
                    continue
            sl, sr = sec[ileft], sec[iright]
            rl, rr = int(si[sl, nVar]), int(si[sr, nVar])
            el, er = int(si[sl, nVar + 1]), int(si[sr, nVar + 1])
            bl, br = int(si[sl, nVar + 2]), int(si[sr, nVar + 2])
            refl, refr = int(bo[ileft, nVar]), int(bo[iright, nVar])
            for isubl in range(bl, bl + rl):                   # :155-192 (1-based)
                var_l = bi[isubl - 1, nVar + 1]
                op_l = bi[isubl - 1, nVar + 2]
                for isubr in range(br, br + rr):
                    var_r = bi[isubr - 1, nVar + 1]
                    op_r = bi[isubr - 1, nVar + 2]
                    if var_r != var_l:
                        continue
                    hit = lookup.get((int(op_l), int(op_r)))   # :171-182, last match wins
                    if hit is None:
                        continue
                    coef, kind = hit
                    im[iright, ileft, kind - 1] += (
                        coef * V[el - 1 + rl * (refl - 1) + (isubl - bl)]
                        * V[er - 1 + rr * (refr - 1) + (isubr - br)])
    return im


def invariant_matrix_for_spectrum(st, ims_prev: np.ndarray) -> np.ndarray:
    """invariantMatrixForSpectrum.F90:71-198 on one rank: <ileft| d^dagger_m |iright> of the
    kept states from the previous iteration's matrix ``ims_prev``."""
    nVar, nb = st.nVar, st.nb
    si, bi, bo, V = st.subspaceInfo, st.basis_input, st.basis_output, st.eigenvector
    new = np.zeros((nb, nb, st.nMat), order="F")
    sec = [_sector_of(si, nVar, bo[i, :nVar]) for i in range(nb)]
    for ileft in range(nb):
        for iright in range(nb):
            diff = bo[ileft, :nVar].astype(np.int64) - bo[iright, :nVar]
            mats = [m for m in range(st.nMat) if np.all(diff == st.cons_diff[m])]   # :111-140
            if not mats:
                continue
            sl, sr = sec[ileft], sec[iright]
            rl, rr = int(si[sl, nVar]), int(si[sr, nVar])
            el, er = int(si[sl, nVar + 1]), int(si[sr, nVar + 1])
            bl, br = int(si[sl, nVar + 2]), int(si[sr, nVar + 2])
            refl, refr = int(bo[ileft, nVar]), int(bo[iright, nVar])
            for isubl in range(bl, bl + rl):                   # :162-196
                op_l = bi[isubl - 1, nVar + 2]
                ref_l = bi[isubl - 1, nVar]
                for isubr in range(br, br + rr):
                    op_r = bi[isubr - 1, nVar + 2]
                    ref_r = bi[isubr - 1, nVar]
                    if op_r != op_l:
                        continue
                    for m in mats:
                        coef = st.cspec[m, op_l - 1]
                        new[iright, ileft, m] += (
                            coef * V[el - 1 + rl * (refl - 1) + (isubl - bl)]
                            * V[er - 1 + rr * (refr - 1) + (isubr - br)]
                            * ims_prev[ref_r - 1, ref_l - 1, m])
    return new


def reduced_density_matrix(st, rdm: np.ndarray, fsi: np.ndarray, point: int) -> Dict[int, float]:
    """reducedDensityMatrix.F90:57-254 on one rank, in place on ``rdm`` (the flat
    reducedDensityMatrix after initializeReducedDensity) and ``fsi`` (fullSubspaceInfo, its
    start_matrix column filled as the loop goes), from pointReducedDensity ``point``.
    Returns the trace of each backward step."""
    nVar, nOps = st.nVar, st.nOps
    FBI, FBO, FV = st.FBI, st.FBO, st.FV
    traces = {}
    for i in range(1, st.nIter - st.startTrancation + 1):
        present = st.nIter - i
        previous = present + 1
        ps = st.mapFull[present] - 1
        qs = st.mapFull[previous] - 1
        for j in range(ps, qs):                                # :88-95
            fsi[j, nVar + 5] = point
            point += int(fsi[j, nVar + 1]) ** 2
        if previous == st.nIter:                               # :168-173
            prev_end = st.elementNumFullSubspace - 1
        else:
            prev_end = st.mapFull[previous + 1] - 2
        diag = 0.0
        for iS in range(ps, qs):                               # :118-254
            n = int(fsi[iS, nVar + 1])
            pout = int(fsi[iS, nVar + 4])
            rho_s = np.zeros((n, n))
            for il in range(n):
                left_index = int(FBO[pout + il - 1, nVar])
                for ir in range(n):
                    right_index = int(FBO[pout + ir - 1, nVar])
                    element = 0.0
                    for op in range(1, nOps + 1):
                        prev_q = fsi[iS, :nVar] - st.operation[op - 1, :nVar]
                        hit = None
                        for iSp in range(qs, prev_end + 1):   # :176-190, first match
                            if np.all(fsi[iSp, :nVar] == prev_q):
                                hit = iSp
                                break
                        if hit is None:
                            continue
                        total = int(fsi[hit, nVar])
                        keep = int(fsi[hit, nVar + 1])
                        pe = int(fsi[hit, nVar + 2])
                        pin = int(fsi[hit, nVar + 3])
                        prm = int(fsi[hit, nVar + 5])
                        ild = ird = None
                        for x in range(pin, pin + total):      # :203-210
                            if FBI[x - 1, nVar + 1] == left_index and FBI[x - 1, nVar + 2] == op:
                                ild = x
                                break
                        for x in range(pin, pin + total):      # :214-220
                            if FBI[x - 1, nVar + 1] == right_index and FBI[x - 1, nVar + 2] == op:
                                ird = x
                                break
                        for k1 in range(1, keep + 1):          # :224-233
                            for k2 in range(1, keep + 1):
                                element += (FV[pe - 1 + (k1 - 1) * total + ild - pin]
                                            * FV[pe - 1 + (k2 - 1) * total + ird - pin]
                                            * rdm[prm - 1 + (k1 - 1) * keep + k2 - 1])
                    rho_s[il, ir] = element
            diag += float(np.trace(rho_s))                     # :243-245
            r0 = int(fsi[iS, nVar + 5])                        # :248-254, row-major
            rdm[r0 - 1:r0 - 1 + n * n] = rho_s.reshape(-1)
        traces[present] = diag
    return traces


def spectrum_element(R: dict, cspec: np.ndarray, nVar: int, start_left: int, start_right: int,
                     max_left: int, max_right: int, var_left: int, var_right: int,
                     ev_left: int, ev_right: int, m: int) -> float:
    """spectrumElement (module.F90:1127-1207): <left column var_left| d^dagger_m |right column
    var_right> by a double loop over the basis states of the two sectors (1-based)."""
    V = R["eigenvector"]
    bi = R["basis_input"]
    ims = R["ims_prev"]
    s2l = ev_left - start_left + max_left * (var_left - 1)
    s2r = ev_right - start_right + max_right * (var_right - 1)
    # the right-hand states of the inner loop (ir), without the zero entries it skips
    r = np.arange(start_right, start_right + max_right)
    vr = V[s2r + r - 1]
    keep = vr != 0.0
    r, vr = r[keep], vr[keep]
    op_r = bi[r - 1, nVar + 2]
    ref_r = bi[r - 1, nVar] - 1
    total = 0.0
    for il in range(start_left, start_left + max_left):
        vl = V[s2l + il - 1]
        if vl == 0.0:
            continue
        op_l = bi[il - 1, nVar + 2]
        ref_l = bi[il - 1, nVar]
        same = op_r == op_l
        # spike_temp: the inner sum over ir of eigenvector_right(ir) * IMS(ref_r, ref_l, m)
        acc = float(np.dot(vr[same], ims[ref_r[same], ref_l - 1, m]))
        if acc == 0.0:
            continue
        total += cspec[m, op_l - 1] * vl * acc
    return total


def _bin(st, container: np.ndarray, energy: float, weight: float, m: int) -> None:
    """binningSpike (module.F90:1210-1254) for one spike."""
    nbin = st.numberOfBin
    off = m * nbin
    if energy == 0.0:
        container[off, 1] += weight
        return
    x = (np.log10(abs(energy)) + 15.0) * 1000.0 + 1.0
    if x <= 0.0:
        container[off, 1] += weight
    elif x >= nbin:
        container[off + nbin - 1, 1] += weight
    else:
        i = max(int(x), 1)            # int() truncates; a reference below 1 becomes 1
        f = x - i
        container[off + i - 1, 1] += (1.0 - f) * weight
        container[off + i, 1] += f * weight


def spike_zero_temperature(st, iteration: int, R: dict, pos: np.ndarray, neg: np.ndarray) -> None:
    """calculateSpectrum.F90:1-151 (spikeZeroTemperature, loop form): adds the T = 0 spikes of
    the last iteration to the weight columns of ``pos`` and ``neg``."""
    nVar = st.nVar
    E, bo, si, nb = R["eigenvalue"], R["basis_output"], R["subspaceInfo"], R["numberOfBasis"]
    gs = [i for i in range(nb) if E[i] < DEGENERACY_THRESHOLD]    # :49-67
    pf = float(len(gs))
    sc = st.scale(iteration)
    for g in gs:
        qg = bo[g, :nVar].astype(np.int64)
        gs_var = int(bo[g, nVar])                                  # :76
        isg = _sector_of(si, nVar, qg)
        dg, eg, bg = int(si[isg, nVar]), int(si[isg, nVar + 1]), int(si[isg, nVar + 2])
        for sign, ops, cont in ((+1, st.pos_op, pos), (-1, st.neg_op, neg)):
            for m in range(st.nMat):
                qe = qg + ops[m]
                ise = _first_sector(si, nVar, qe)
                if ise is None:
                    continue
                de, ee, be = int(si[ise, nVar]), int(si[ise, nVar + 1]), int(si[ise, nVar + 2])
                for iexs in range(be, be + de):
                    ex_var = int(bo[iexs - 1, nVar])
                    if sign > 0:                                   # :106-117
                        s = spectrum_element(R, st.cspec, nVar, be, bg, de, dg, ex_var, gs_var, ee, eg, m)
                    else:                                          # :135-146
                        s = spectrum_element(R, st.cspec, nVar, bg, be, dg, de, gs_var, ex_var, eg, ee, m)
                    _bin(st, cont, sign * E[iexs - 1] * sc, s * s / pf, m)


def _first_sector(si, nVar, qn) -> Optional[int]:
    """findSubspace (module.F90:1256-1284): first match."""
    for isub in range(si.shape[0]):
        if all(int(qn[v]) == int(si[isub, v]) for v in range(nVar)):
            return isub
    return None


def spike_cfs(st, iteration: int, nb_full: int, R: dict, pos: np.ndarray, neg: np.ndarray) -> List[float]:
    """calculateSpectrum.F90:153-535 (spikeCFS, loop form) on one rank and one thread: adds the
    CFS spikes of the discarded states of this iteration to ``pos`` and ``neg``; returns the
    raw sums (negative then positive, per matrix type) of the binned-vs-raw check."""
    nVar = st.nVar
    E, bo, si, nb = R["eigenvalue"], R["basis_output"], R["subspaceInfo"], R["numberOfBasis"]
    FSI = st.FSI
    f0 = st.mapFull[iteration] - 1
    f1 = st.mapFull[iteration + 1] - 1
    sc = st.scale(iteration)
    tot_neg = [0.0] * st.nMat
    tot_pos = [0.0] * st.nMat
    rdm = st.rdm

    def find_full(q):                     # findFullSubspace (module.F90:1286-1314)
        for j in range(f0, f1):
            if np.all(FSI[j, :nVar] == q):
                return j
        return None

    def start_output(q):                  # findStartOutput (module.F90:1316-1338)
        for i in range(nb):
            if np.all(bo[i, :nVar] == q):
                return i + 1
        return None

    for il in range(nb + 1, nb_full + 1):                          # :281
        l_var = int(bo[il - 1, nVar])
        El = E[il - 1]
        ql = bo[il - 1, :nVar].astype(np.int64)
        isl = _first_sector(si, nVar, ql)
        dl, elv, bl = int(si[isl, nVar]), int(si[isl, nVar + 1]), int(si[isl, nVar + 2])
        for part, ops in ((0, st.pos_op), (1, st.neg_op)):
            for m in range(st.nMat):
                qk = ql + ops[m]
                fk = find_full(qk)
                isk = _first_sector(si, nVar, qk)
                if fk is None or isk is None:
                    continue
                sbo = start_output(qk)
                kk = int(FSI[fk, nVar + 1])
                pm = int(FSI[fk, nVar + 5])
                dk, ek, bk = int(si[isk, nVar]), int(si[isk, nVar + 1]), int(si[isk, nVar + 2])
                spike = []
                for ik in range(1, kk + 1):                        # :326-331, :395-400
                    k_var = int(bo[sbo + ik - 2, nVar])
                    if part == 0:
                        spike.append(spectrum_element(R, st.cspec, nVar, bk, bl, dk, dl, k_var, l_var, ek, elv, m))
                    else:
                        spike.append(spectrum_element(R, st.cspec, nVar, bl, bk, dl, dk, l_var, k_var, elv, ek, m))
                for ik1 in range(sbo, sbo + kk):                   # :334-352, :403-420
                    k1_var = int(bo[ik1 - 1, nVar])
                    Ek1 = E[ik1 - 1]
                    w = 0.0
                    s1 = spike[ik1 - sbo]
                    for ik2 in range(sbo, sbo + kk):
                        k2_var = int(bo[ik2 - 1, nVar])
                        w += s1 * spike[ik2 - sbo] * rdm[pm - 1 + kk * (k2_var - 1) + (k1_var - 1)]
                    if part == 0:
                        tot_neg[m] += w
                        _bin(st, neg, (Ek1 - El) * sc, w, m)
                    else:
                        tot_pos[m] += w
                        _bin(st, pos, (El - Ek1) * sc, w, m)
    return tot_neg + tot_pos
