"""restart.dat through the drop-in replay on the GPU (nrg_run with host_drop_in = 1):
the library's file is the reference-semantics state (the oracle's loader resumes from it
and finishes with the oracle's spectrum), and the library resumes from a file the oracle
wrote for an interrupted run.

Tolerances as in the routine parity tests: bins within 1e-8 absolute, kept counts and the
integer tables of the file identical, eigenvalues within 1e-12 relative."""
import numpy as np
import pytest

from oracle import nrg_oracle as O
from nrg_b200 import NrgError, model

from helpers import small_siam, write_case

pytestmark = pytest.mark.gpu

BIN_TOL = 1e-8


@pytest.fixture(scope="module")
def case(tmp_path_factory):
    d = write_case(small_siam(n_keep=48, n_iterations=14), str(tmp_path_factory.mktemp("gpu_restart")))
    return d, O.run(d)


def _bins_diff(binPos, binNeg, st):
    return max(float(np.max(np.abs(binPos[:, 1] - st.binPos[:, 1]))),
               float(np.max(np.abs(binNeg[:, 1] - st.binNeg[:, 1]))))


def test_library_file_resumes_in_the_oracle(case, ctx_factory, tmp_path):
    d, full = case
    ctx = ctx_factory(model.read_inputs(d))
    lib = str(tmp_path / "lib.dat")
    res = ctx.run(spectrum=True, host_drop_in=True, restart_file=lib, save_restart=True)
    assert _bins_diff(res["binPos"], res["binNeg"], full) <= BIN_TOL
    # the last write precedes the last CFS step: the oracle finishes the loop from it
    st = O.run_with_restart(d, load_path=lib)
    assert _bins_diff(st.binPos, st.binNeg, full) <= BIN_TOL
    # the oracle's own file for the same step: same integer tables and eigenvalues
    ref = str(tmp_path / "oracle.dat")
    O.run_with_restart(d, save_path=ref, stop_before=full.nIter)
    a, b = O.State(d), O.State(d)
    assert O.load_restart(a, lib) == O.load_restart(b, ref) == full.nIter
    assert np.array_equal(a.FSI, b.FSI) and a.mapFull == b.mapFull
    assert (a.startTrancation, a.flag_truncation) == (b.startTrancation, b.flag_truncation)
    for it in range(full.first, full.nIter + 1):
        ra, rb = a.restore[it], b.restore[it]
        for key in ("subspaceInfo", "basis_input"):
            assert np.array_equal(ra[key], rb[key]), (it, key)
        # basis_output: the kept states in index order are identical; the discarded ones
        # follow in energy order (postprocess.F90:143-160), where exactly degenerate
        # states may change places with last-bit differences of the eigenvalues
        nb = rb["numberOfBasis"]
        assert ra["numberOfBasis"] == nb
        assert np.array_equal(ra["basis_output"][:nb], rb["basis_output"][:nb]), it
        ta, tb = ra["basis_output"][nb:], rb["basis_output"][nb:]
        assert np.array_equal(ta[np.lexsort(ta.T[::-1])], tb[np.lexsort(tb.T[::-1])]), it
        assert ra["eigenvector"].size == rb["eigenvector"].size
        e = rb["eigenvalue"]
        assert np.max(np.abs(ra["eigenvalue"] - e) / np.maximum(1.0, np.abs(e))) <= 1e-12
    assert a.rdm.size == b.rdm.size
    assert open(lib, "rb").read()[:88] == open(ref, "rb").read()[:88]   # mode, step, hami


@pytest.mark.parametrize("step", ["start", "middle"])
def test_library_resumes_an_interrupted_oracle_run(case, ctx_factory, tmp_path, step):
    d, full = case
    k = full.startTrancation if step == "start" else (full.startTrancation + full.nIter) // 2
    path = str(tmp_path / "restart.dat")
    O.run_with_restart(d, save_path=path, stop_before=k)
    ctx = ctx_factory(model.read_inputs(d))
    res = ctx.run(spectrum=True, host_drop_in=True, restart_file=path, load_restart=True)
    assert _bins_diff(res["binPos"], res["binNeg"], full) <= BIN_TOL
    its = list(range(full.first, full.nIter + 1))
    assert [int(x) for x in res["kept"]] == [full.restore[i]["numberOfBasis"] for i in its]
    assert res["startTrancation"] == full.startTrancation
    # resuming with saving on rewrites the file before every later step
    keep = str(tmp_path / "resume_and_save.dat")
    O.run_with_restart(d, save_path=keep, stop_before=k)
    res2 = ctx.run(spectrum=True, host_drop_in=True, restart_file=keep, load_restart=True, save_restart=True)
    assert _bins_diff(res2["binPos"], res2["binNeg"], full) <= BIN_TOL
    st = O.State(d)
    assert O.load_restart(st, keep) == (full.nIter if k < full.nIter else k)


def test_restart_errors(case, ctx_factory, tmp_path):
    d, full = case
    ctx = ctx_factory(model.read_inputs(d))
    with pytest.raises(NrgError):   # loadRestart: "restart file not found"
        ctx.run(spectrum=True, host_drop_in=True, restart_file=str(tmp_path / "missing.dat"), load_restart=True)
    path = tmp_path / "broken.dat"
    O.run_with_restart(d, save_path=str(path), stop_before=full.startTrancation)
    raw = bytearray(path.read_bytes())
    raw[0:4] = np.array([1001], dtype="<i4").tobytes()
    path.write_bytes(bytes(raw))
    with pytest.raises(NrgError):   # "broken restart file"
        ctx.run(spectrum=True, host_drop_in=True, restart_file=str(path), load_restart=True)
    with pytest.raises(NrgError):   # device-resident runs keep no restore stock on the host
        ctx.run(spectrum=True, restart_file=str(tmp_path / "x.dat"), save_restart=True)
    # a truncated file is refused, not read past its end
    good = tmp_path / "good.dat"
    O.run_with_restart(d, save_path=str(good), stop_before=full.startTrancation)
    short = tmp_path / "short.dat"
    short.write_bytes(good.read_bytes()[:-100])
    with pytest.raises(NrgError):
        ctx.run(spectrum=True, host_drop_in=True, restart_file=str(short), load_restart=True)
    # the context stays usable
    res = ctx.run(spectrum=True, host_drop_in=True)
    assert _bins_diff(res["binPos"], res["binNeg"], full) <= BIN_TOL
