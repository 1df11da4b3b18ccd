"""Full-density-matrix spectrum at T > 0 (device-resident run) against the oracle's FDM
restatement, which is pinned by its T -> 0 limit (the CFS spectrum), a finite-T
non-interacting known answer and its sum rules (tests/test_oracle.py).

Tolerances: bins 1e-8 absolute; sum rule 1e-10; trace of every shell (kept-space trace
plus the weight discarded up to it) 1e-12."""
import numpy as np
import pytest

from oracle import nrg_oracle as O
from nrg_b200 import model

from helpers import small_siam, write_case

pytestmark = pytest.mark.gpu

BIN_TOL = 1e-8
SUM_TOL = 1e-10


@pytest.fixture(scope="module")
def case(ctx_factory):
    inp = small_siam(n_keep=48, n_iterations=14)
    d = write_case(inp)
    st = O.run(d)
    ctx = ctx_factory(model.read_inputs(d))
    return st, ctx


@pytest.mark.parametrize("factor", [0.1, 3.0])
def test_fdm_matches_oracle(case, factor):
    st, ctx = case
    T = factor * st.scale(st.nIter)
    bp, bn, diag = O.fdm_spectrum(st, T)
    res = ctx.run(spectrum=True, temperature=T)
    assert np.max(np.abs(res["binPos"][:, 1] - bp[:, 1])) <= BIN_TOL
    assert np.max(np.abs(res["binNeg"][:, 1] - bn[:, 1])) <= BIN_TOL
    nbin = st.numberOfBin
    for m in range(st.nMat):
        tot = res["binPos"][m * nbin:(m + 1) * nbin, 1].sum() + res["binNeg"][m * nbin:(m + 1) * nbin, 1].sum()
        assert abs(tot - 1.0) <= SUM_TOL
    tr = [res["rdmTrace"][N] for N in range(st.startTrancation, st.nIter)]
    assert max(abs(t - 1.0) for t in tr) <= 1e-12


def test_fdm_zero_temperature_limit_on_the_device(case):
    st, ctx = case
    res = ctx.run(spectrum=True, temperature=1e-3 * st.scale(st.nIter))
    assert np.max(np.abs(res["binPos"][:, 1] - st.binPos[:, 1])) <= BIN_TOL
    assert np.max(np.abs(res["binNeg"][:, 1] - st.binNeg[:, 1])) <= BIN_TOL


def test_fdm_two_orbital_model(ctx_factory):
    inp = model.two_orbital_hund(n_keep=96, n_iterations=7)
    d = write_case(inp)
    st = O.run(d)
    ctx = ctx_factory(model.read_inputs(d))
    T = 0.5 * st.scale(st.nIter)
    bp, bn, _ = O.fdm_spectrum(st, T)
    res = ctx.run(spectrum=True, temperature=T)
    assert np.max(np.abs(res["binPos"][:, 1] - bp[:, 1])) <= BIN_TOL
    assert np.max(np.abs(res["binNeg"][:, 1] - bn[:, 1])) <= BIN_TOL
