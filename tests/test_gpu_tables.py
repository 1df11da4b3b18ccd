"""Per-state bookkeeping of the device-resident run on the device (tables.cu): the
truncation of postprocess.F90:69-140 by radix selection, and the basis records and
(sector, operation) row lists of prepareBasis.F90:31-114 written per row from
sector-level runs.

With NRG_CHECK_TABLES=1 the run compares, at every iteration, the device's kept counts
with the host's truncation of the same eigenvalues, and the device's sector table, records
and row lists with the host's prepareBasis of the same kept states (the host code is
bit-exact against the oracle on the CPU: tests/test_prepare_basis.py, test_truncate.py);
any difference fails the run.  The same model is then run with the bookkeeping on the
host (NRG_HOST_TABLES=1) and against the oracle.  The cases: a SIAM, a particle-hole
asymmetric bath, a non-interacting impurity whose degenerate levels make the truncation
cut back by 0.001 steps at every other iteration, and the N_keep = 2048 workload's first
iterations (sectors of the bench's sizes).
"""
import os

import numpy as np
import pytest

from oracle import nrg_oracle as O
from nrg_b200 import model

from helpers import small_siam, write_case

pytestmark = pytest.mark.gpu

BIN_TOL = 1e-8

CASES = {
    "siam": lambda: small_siam(n_keep=64, n_iterations=16),
    "bath": lambda: model.siam_bath(U=0.2, eps_d=-0.07, hybridization=lambda e: 0.02 * (1.0 + 0.4 * e),
                                    Lambda=2.5, n_keep=64, n_iterations=14),
    "cut_back": lambda: model.siam(U=0.0, Gamma=0.01, eps_d=0.0, Lambda=2.5, n_keep=40, n_iterations=14),
    "n_keep_2048": lambda: model.config(2, n_iterations=10),
}


@pytest.fixture
def env():
    saved = {k: os.environ.get(k) for k in ("NRG_CHECK_TABLES", "NRG_HOST_TABLES")}
    yield os.environ
    for k, v in saved.items():
        if v is None:
            os.environ.pop(k, None)
        else:
            os.environ[k] = v


@pytest.mark.parametrize("case", list(CASES))
def test_device_tables_equal_the_host_bookkeeping(case, ctx_factory, env):
    d = write_case(CASES[case]())
    ctx = ctx_factory(model.read_inputs(d))
    env["NRG_CHECK_TABLES"] = "1"
    env.pop("NRG_HOST_TABLES", None)
    dev = ctx.run(spectrum=True)             # fails on the first table that differs
    env.pop("NRG_CHECK_TABLES")
    env["NRG_HOST_TABLES"] = "1"
    host = ctx.run(spectrum=True)
    env.pop("NRG_HOST_TABLES")
    assert [int(k) for k in dev["kept"]] == [int(k) for k in host["kept"]]
    assert dev["startTrancation"] == host["startTrancation"]
    f, g = np.nan_to_num(dev["flow"]), np.nan_to_num(host["flow"])
    assert np.max(np.abs(f - g) / np.maximum(1.0, np.abs(g))) <= 1e-12
    assert np.max(np.abs(dev["binPos"][:, 1] - host["binPos"][:, 1])) <= 1e-12
    assert np.max(np.abs(dev["binNeg"][:, 1] - host["binNeg"][:, 1])) <= 1e-12
    if case == "n_keep_2048":
        return                               # the whole workload is pinned by its golden fixture
    st = O.run(d)
    its = list(range(st.first, st.nIter + 1))
    assert [int(k) for k in dev["kept"]] == [st.kept[i] for i in its]
    if case == "cut_back":
        assert any(st.kept[i] < 40 for i in its[1:-1])   # the cut-back ran
    assert np.max(np.abs(dev["binPos"][:, 1] - st.binPos[:, 1])) <= BIN_TOL
    assert np.max(np.abs(dev["binNeg"][:, 1] - st.binNeg[:, 1])) <= BIN_TOL


def test_device_tables_move_only_sector_level_data(ctx_factory, env):
    """Host-to-device bytes of a forward sweep: the per-state records and row lists of
    every iteration after the first no longer cross."""
    inp = model.config(2, n_iterations=10)
    d = write_case(inp)
    ctx = ctx_factory(model.read_inputs(d))
    moved = {}
    for mode in ("device", "host"):
        env.pop("NRG_HOST_TABLES", None)
        if mode == "host":
            env["NRG_HOST_TABLES"] = "1"
        res = ctx.run(spectrum=False)
        ctx.reset_stats()
        res = ctx.run(spectrum=False)
        moved[mode] = ctx.stats()["h2d_bytes"]
    env.pop("NRG_HOST_TABLES", None)
    rs = inp.numberOfVariation + 3
    records = sum(4 * (rs + 1) * int(nb) for nb in res["numberOfBasisFull"][1:])
    print(f"host-to-device bytes per sweep: device tables {moved['device']}, host tables {moved['host']}, "
          f"records and row lists {records}")
    assert moved["host"] - moved["device"] >= 0.75 * records, moved   # less the runs and sector tables
