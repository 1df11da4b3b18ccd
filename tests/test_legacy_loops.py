"""The oracle's DGEMM form against its second form, the reference's loop-form routines.

``oracle/legacy_loops.py`` restates invariantMatrix.F90, invariantMatrixForSpectrum.F90,
reducedDensityMatrix.F90 and calculateSpectrum.F90 (with spectrumElement) element by
element.  A whole oracle run is made with the loop form computed beside every DGEMM-form
routine on the same state; the two must agree to 1e-13 (absolute: invariant matrices,
density matrices and spectral weights are all of order one or smaller), which pins the
eigenvector indexing (column-major columns, read with column semantics where the DGEMM
routines' slice bounds are garbled), the sector lookups, the density-matrix storage order
and the spike energies of the DGEMM oracle that the GPU tests compare with.
"""
import numpy as np
import pytest

from oracle import legacy_loops as LL
from oracle import nrg_oracle as O
from nrg_b200 import model

from helpers import small_siam, write_case

TOL = 1e-13


def _run_both(d, monkeypatch):
    err = dict(im=0.0, ims=0.0, rdm=0.0, trace=0.0, bins=0.0, raw=0.0)
    calls = dict(im=0, ims=0, rdm=0, spike0=0, cfs=0)
    im_dgemm = O.invariant_matrix_dgemm
    ims_dgemm = O.invariant_matrix_for_spectrum_dgemm
    rdm_dgemm = O.reduced_density_matrix_calculation
    cfs = O.cfs_spectrum_calculation

    def im_both(st, it):
        im_dgemm(st, it)
        err["im"] = max(err["im"], float(np.max(np.abs(LL.invariant_matrix(st) - st.im), initial=0.0)))
        calls["im"] += 1

    def ims_both(st, it):
        prev = st.ims
        ims_dgemm(st, it)
        loop = LL.invariant_matrix_for_spectrum(st, prev)
        err["ims"] = max(err["ims"], float(np.max(np.abs(loop - st.ims), initial=0.0)))
        calls["ims"] += 1

    def rdm_both(st):
        rdm0, fsi0, p0 = st.rdm.copy(), st.FSI.copy(), st.pointReducedDensity
        rdm_dgemm(st)
        traces = LL.reduced_density_matrix(st, rdm0, fsi0, p0)
        assert np.array_equal(fsi0, st.FSI)          # start_matrix of every sector
        err["rdm"] = float(np.max(np.abs(rdm0 - st.rdm)))
        err["trace"] = max(abs(traces[N] - st.rdm_trace[N]) for N in traces)
        calls["rdm"] += 1

    def cfs_both(st, it, literal=False):
        p0, n0 = st.binPos[:, 1].copy(), st.binNeg[:, 1].copy()
        cfs(st, it, literal=literal)
        R = O.get_restore(st, it)
        pos, neg = np.zeros_like(st.binPos), np.zeros_like(st.binNeg)
        if it == st.nIter:
            LL.spike_zero_temperature(st, it, R, pos, neg)
            calls["spike0"] += 1
        else:
            raw = LL.spike_cfs(st, it, R["numberOfBasis_full"], R, pos, neg)
            # the reference's own check: the binned sums equal the raw sums
            nbin = st.numberOfBin
            for m in range(st.nMat):
                err["raw"] = max(err["raw"], abs(neg[m * nbin:(m + 1) * nbin, 1].sum() - raw[m]),
                                 abs(pos[m * nbin:(m + 1) * nbin, 1].sum() - raw[st.nMat + m]))
            calls["cfs"] += 1
        err["bins"] = max(err["bins"], float(np.max(np.abs(pos[:, 1] - (st.binPos[:, 1] - p0)))),
                          float(np.max(np.abs(neg[:, 1] - (st.binNeg[:, 1] - n0)))))

    monkeypatch.setattr(O, "invariant_matrix_dgemm", im_both)
    monkeypatch.setattr(O, "invariant_matrix_for_spectrum_dgemm", ims_both)
    monkeypatch.setattr(O, "reduced_density_matrix_calculation", rdm_both)
    monkeypatch.setattr(O, "cfs_spectrum_calculation", cfs_both)
    st = O.run(d)
    return st, err, calls


@pytest.mark.parametrize("case", ["siam", "two_orbital"])
def test_loop_form_equals_dgemm_form(case, monkeypatch):
    if case == "siam":
        # truncated from iteration 2 on; particle-hole asymmetric, so no accidental zeros
        inp = small_siam(n_keep=24, n_iterations=7, U=0.1, Gamma=0.01, eps_d=-0.03)
    else:
        # 16 local states, two chains, tied sort keys; iterations -1..1, truncated at 0
        inp = model.two_orbital_hund(U=0.2, J=0.02, Gamma=0.015, Lambda=3.0, n_keep=8, n_iterations=3)
    st, err, calls = _run_both(write_case(inp), monkeypatch)
    assert st.flag_truncation
    assert calls["im"] == calls["ims"] == st.nIter - st.first
    assert calls["rdm"] == 1 and calls["spike0"] == 1 and calls["cfs"] == st.nIter - st.startTrancation
    for k in ("im", "ims", "rdm", "trace", "bins", "raw"):
        assert err[k] <= TOL, (k, err[k])
