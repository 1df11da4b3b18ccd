"""Independent instances side by side on one GPU (nrg_run_batch): every instance of a small
sweep matches its own oracle run, as it does when run alone.

Tolerances as in the routine parity tests: kept counts identical, spectral bins within
1e-8 absolute, sum rule within 1e-10."""
import numpy as np
import pytest

from oracle import nrg_oracle as O
from nrg_b200 import Context, NrgError, model, run_batch, sweep

from helpers import write_case

pytestmark = pytest.mark.gpu

BIN_TOL = 1e-8
SUM_TOL = 1e-10


def _small_sweep():
    xs = sweep.sweep_instances(count=5, seed=11, n_iterations=12, nkeep_choices=(24, 32, 48))
    return sorted(xs, key=lambda x: (-x.cost(), x.index))


def test_batch_matches_oracle_per_instance():
    xs = _small_sweep()
    dirs = [write_case(x.build()) for x in xs]
    ref = [O.run(d) for d in dirs]
    ctxs = []
    try:
        for d in dirs:
            c = Context(0)
            c.set_model(model.read_inputs(d))
            ctxs.append(c)
        for _ in range(2):   # a second batch reuses every context's device storage
            results, statuses = run_batch(ctxs, spectrum=True, concurrency=3)
            assert statuses == [0] * len(xs)
            for st, res in zip(ref, results):
                its = list(range(st.first, st.nIter + 1))
                assert [int(k) for k in res["kept"]] == [st.kept[i] for i in its]
                assert np.max(np.abs(res["binPos"][:, 1] - st.binPos[:, 1])) <= BIN_TOL
                assert np.max(np.abs(res["binNeg"][:, 1] - st.binNeg[:, 1])) <= BIN_TOL
                nbin = st.numberOfBin
                for m in range(st.nMat):
                    tot = (res["binPos"][m * nbin:(m + 1) * nbin, 1].sum()
                           + res["binNeg"][m * nbin:(m + 1) * nbin, 1].sum())
                    assert abs(tot - 1.0) <= SUM_TOL
    finally:
        for c in ctxs:
            c.close()


def test_batch_fdm_matches_the_instances_run_alone():
    """The full-density-matrix spectrum (the many-instance workload's T > 0) side by side:
    each instance's bins and shell traces equal its run alone (the same kernels on the
    same data; FP64 atomics in the binning allow last-bit differences)."""
    xs = _small_sweep()[:3]
    T = 1e-4
    ctxs = []
    try:
        for x in xs:
            c = Context(0)
            c.set_model(x.build())
            ctxs.append(c)
        alone = [c.run(spectrum=True, temperature=T) for c in ctxs]
        results, statuses = run_batch(ctxs, spectrum=True, concurrency=3, temperature=T)
        assert statuses == [0] * len(xs)
        for a, r in zip(alone, results):
            assert [int(k) for k in r["kept"]] == [int(k) for k in a["kept"]]
            assert np.max(np.abs(r["binPos"][:, 1] - a["binPos"][:, 1])) <= 1e-12
            assert np.max(np.abs(r["binNeg"][:, 1] - a["binNeg"][:, 1])) <= 1e-12
            assert np.nanmax(np.abs(r["rdmTrace"] - a["rdmTrace"])) <= 1e-12
            nbin = r["numberOfBin"]
            for m in range(2):
                tot = (r["binPos"][m * nbin:(m + 1) * nbin, 1].sum() + r["binNeg"][m * nbin:(m + 1) * nbin, 1].sum())
                assert abs(tot - 1.0) <= SUM_TOL
    finally:
        for c in ctxs:
            c.close()


def test_batch_rejects_a_repeated_context():
    inp = _small_sweep()[0].build()
    c = Context(0)
    try:
        c.set_model(inp)
        with pytest.raises(NrgError):
            run_batch([c, c], spectrum=False)
    finally:
        c.close()
