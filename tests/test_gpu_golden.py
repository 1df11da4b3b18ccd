"""Whole runs of the benchmarked workloads against the committed golden fixtures.

The fixtures (``tests/golden/*.npz``, written by ``tests/golden/make_golden.py`` from the
CPU oracle) hold, per iteration, the kept count, the state count before truncation, the
ground-state energy, the 64 lowest kept energies and calcThermo's (Cn, Sn, Xn), the
density-matrix trace of every backward step, and the nonzero spectral bins:

* the N_keep = 2048 SIAM workload, all 60 iterations with density matrices and the T = 0
  CFS spectrum (the second bench object);
* the N_keep = 4096 SIAM workload (the bench headline), all 60 iterations with density
  matrices and the T = 0 CFS spectrum;
* the two-orbital Hund model at N_keep = 8192 (16 local states), its first 5 iterations
  (-1..3), forward sweep only: 131,104 states at iteration 3 in sectors of order up to
  ~8,800, past the cluster tridiagonalisation's and the shared-memory back-transformation's
  size limits, with tied sort keys in prepareBasis.

Both the device-resident run and the drop-in replay (every routine through its entry point
with host arrays, page-locked, and for the N_keep = 4096 case also pageable) are compared.  Tolerances: kept counts and state counts equal (the
truncation edge with its degenerate multiplets, postprocess.F90:79-126, is where a
bit-level eigenvalue difference would show); energies <= 1e-11 * max(1, |E|); thermo
<= 1e-11 relative; density-matrix traces 1e-12; bins <= 1e-8 absolute; sum rule 1e-10.
A last test compares the invariant matrices of one full-size iteration of the N_keep =
2048 workload, routine against routine, on identical inputs (1e-12 absolute).
"""
import os

import numpy as np
import pytest

from oracle import nrg_oracle as O
from nrg_b200 import model

from helpers import write_case

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
E_TOL = 1e-11
THERMO_TOL = 1e-11
TRACE_TOL = 1e-12
BIN_TOL = 1e-8
SUM_TOL = 1e-10
MAT_TOL = 1e-12

CASES = {
    "siam_nkeep2048": lambda: model.config(2),
    "siam_nkeep4096": lambda: model.config(3),
}


def _golden(name):
    return dict(np.load(os.path.join(HERE, "golden", name + ".npz")))


def _bins(g, key, n):
    w = np.zeros(n)
    w[g[key + "_index"]] = g[key + "_weight"]
    return w


def _compare_forward(res, g, device_resident):
    assert np.array_equal(np.asarray(res["kept"], dtype=np.int32), g["kept"])
    assert np.array_equal(np.asarray(res["numberOfBasisFull"], dtype=np.int32), g["numberOfBasisFull"])
    gse = g["groundStateEnergy"]
    assert np.max(np.abs(res["groundStateEnergy"] - gse) / np.maximum(1.0, np.abs(gse))) <= E_TOL
    flow = g["flow"]
    ok = ~np.isnan(flow)
    got = res["flow"][:, :flow.shape[1]]
    assert np.max(np.abs(got[ok] - flow[ok]) / np.maximum(1.0, np.abs(flow[ok]))) <= E_TOL
    if device_resident:
        th = g["thermo"]
        assert np.max(np.abs(res["thermo"] - th) / np.maximum(1.0, np.abs(th))) <= THERMO_TOL


def _compare(res, g, device_resident):
    assert int(res["startTrancation"]) == int(g["startTrancation"])
    assert np.array_equal(np.asarray(res["kept"], dtype=np.int32), g["kept"])
    assert np.array_equal(np.asarray(res["numberOfBasisFull"], dtype=np.int32), g["numberOfBasisFull"])
    gse = g["groundStateEnergy"]
    assert np.max(np.abs(res["groundStateEnergy"] - gse) / np.maximum(1.0, np.abs(gse))) <= E_TOL
    flow = g["flow"]
    ok = ~np.isnan(flow)
    got = res["flow"][:, :flow.shape[1]]
    assert np.max(np.abs(got[ok] - flow[ok]) / np.maximum(1.0, np.abs(flow[ok]))) <= E_TOL
    if device_resident:
        th = g["thermo"]
        assert np.max(np.abs(res["thermo"] - th) / np.maximum(1.0, np.abs(th))) <= THERMO_TOL
        tr = g["rdmTrace"]
        m = ~np.isnan(tr)
        assert np.max(np.abs(res["rdmTrace"][m] - tr[m])) <= TRACE_TOL
    nbin, nmat = int(g["numberOfBin"]), int(g["nMat"])
    assert int(res["numberOfBin"]) == nbin
    for key, arr in (("binPos", res["binPos"]), ("binNeg", res["binNeg"])):
        assert np.max(np.abs(arr[:, 1] - _bins(g, key, nbin * nmat))) <= BIN_TOL
    for m in range(nmat):
        tot = res["binPos"][m * nbin:(m + 1) * nbin, 1].sum() + res["binNeg"][m * nbin:(m + 1) * nbin, 1].sum()
        assert abs(tot - 1.0) <= SUM_TOL


@pytest.mark.parametrize("name", list(CASES))
def test_whole_run_matches_golden(ctx_factory, name):
    g = _golden(name)
    ctx = ctx_factory(CASES[name]())
    res = ctx.run(spectrum=True, flow_stride=64)
    _compare(res, g, device_resident=True)
    res2 = ctx.run(spectrum=True, flow_stride=64, host_drop_in=True)
    _compare(res2, g, device_resident=False)
    if name == "siam_nkeep4096":
        # the caller's module arrays in pageable memory (a Fortran allocatable): the routines
        # gather the runs they read on the host instead of reading pinned memory directly
        res3 = ctx.run(spectrum=True, flow_stride=64, host_drop_in=True, host_pageable=True)
        _compare(res3, g, device_resident=False)
    ctx.release_storage()


def _two_orbital_window():
    inp = model.config(4, n_iterations=5)
    inp.flag_spectrum = False
    return inp


def test_two_orbital_window_matches_golden(ctx_factory):
    g = _golden("two_orbital_nkeep8192_n5")
    ctx = ctx_factory(_two_orbital_window())
    res = ctx.run(spectrum=False, flow_stride=64)
    _compare_forward(res, g, device_resident=True)
    res2 = ctx.run(spectrum=False, flow_stride=64, host_drop_in=True)
    _compare_forward(res2, g, device_resident=False)
    ctx.release_storage()


def test_invariant_matrices_full_size_iteration(ctx_factory):
    # iteration 5 of the N_keep = 2048 workload: ~9,800 states before truncation, ~2,450 kept
    inp = model.config(2, n_iterations=8)
    d = write_case(inp)
    st = O.State(d)
    ctx = ctx_factory(model.read_inputs(d))
    it = 5
    for i in range(st.first, it):
        O.nrg_iteration(st, i)
    O.prepare_basis(st, it)
    si, bi = st.subspaceInfo.copy(), st.basis_input.copy()
    O.diagonalization(st, it)
    st.thermo[it] = O.calc_thermo(st)
    O.truncate(st, it)
    assert st.nb >= 2048 and st.numberOfBasis_full > 8000
    ims_old = st.ims.copy(order="F")
    im_g = ctx.invariant_matrix_dgemm(it, si, bi, st.nb, st.basis_output, st.eigenvector)
    ims_g = ctx.invariant_matrix_for_spectrum_dgemm(it, si, bi, st.nb, st.basis_output, st.eigenvector, ims_old)
    O.invariant_matrix_dgemm(st, it)
    O.invariant_matrix_for_spectrum_dgemm(st, it)
    assert float(np.max(np.abs(im_g - st.im))) <= MAT_TOL
    assert float(np.max(np.abs(ims_g - st.ims))) <= MAT_TOL
