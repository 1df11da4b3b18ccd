"""restart.dat of the CFS phase on the CPU: the oracle's restatement of saveRestart /
loadRestart (module.F90:1710-1890) and of the restart branch of main.F90:165-224.

An interrupted run (the file written for CFS step k, then nothing) resumed from the file
must give the bins of the uninterrupted run; the file's words follow saveRestart's write
list (Fortran stream output: no record markers, 4-byte integers, 8-byte reals)."""
import numpy as np
import pytest

from oracle import nrg_oracle as O
from nrg_b200 import model

from helpers import small_siam, write_case


@pytest.fixture(scope="module")
def case(tmp_path_factory):
    d = write_case(small_siam(n_keep=48, n_iterations=14), str(tmp_path_factory.mktemp("restart")))
    return d, O.run(d)


@pytest.fixture(scope="module")
def two_orbital(tmp_path_factory):
    d = write_case(model.two_orbital_hund(n_keep=96, n_iterations=6), str(tmp_path_factory.mktemp("restart2")))
    return d, O.run(d)


def test_two_orbital_resume_gives_the_full_spectrum(two_orbital, tmp_path):
    # four matrix types, tied basis records, truncation from the second iteration on
    d, full = two_orbital
    assert full.nMat == 4 and full.startTrancation < full.nIter
    for k in range(full.startTrancation, full.nIter + 1):
        path = str(tmp_path / f"restart_{k}.dat")
        O.run_with_restart(d, save_path=path, stop_before=k)
        st = O.run_with_restart(d, load_path=path)
        assert np.array_equal(st.binPos, full.binPos) and np.array_equal(st.binNeg, full.binNeg)


def test_resume_from_an_interrupted_cfs_loop_gives_the_full_spectrum(case, tmp_path):
    d, full = case
    assert full.startTrancation < full.nIter - 2
    for k in (full.startTrancation, full.startTrancation + 2, full.nIter):
        path = str(tmp_path / f"restart_{k}.dat")
        O.run_with_restart(d, save_path=path, stop_before=k)
        st = O.run_with_restart(d, load_path=path)
        assert np.array_equal(st.binPos, full.binPos) and np.array_equal(st.binNeg, full.binNeg)


def test_resumed_run_rewrites_the_file_after_its_step(case, tmp_path):
    # load at step k with saving on: the file then holds the state before the last step
    d, full = case
    k = full.startTrancation + 1
    a = str(tmp_path / "a.dat")
    O.run_with_restart(d, save_path=a, stop_before=k)
    O.run_with_restart(d, load_path=a, save_path=a)
    st = O.State(d)
    assert O.load_restart(st, a) == full.nIter
    b = str(tmp_path / "b.dat")
    O.run_with_restart(d, save_path=b, stop_before=full.nIter)
    assert open(a, "rb").read() == open(b, "rb").read()


def test_file_layout_follows_the_write_list(case, tmp_path):
    d, full = case
    k = full.startTrancation + 2
    path = str(tmp_path / "r.dat")
    O.run_with_restart(d, save_path=path, stop_before=k)
    raw = open(path, "rb").read()
    w = np.frombuffer(raw[:4 * 24], dtype="<i4")
    assert w[0] == 1002 and w[1] == k                          # MODE_RESTART_CFS, iteration
    hami = w[2:22]
    assert hami[0] == full.nIter and hami[2] == full.nVar and hami[12] == full.nOps
    assert hami[14] == full.first and hami[17] == full.startTrancation and hami[18] == 1
    assert hami[9] == full.restore[k - 1]["numberOfBasis"]     # after getRestore(k-1)
    assert w[22] == full.first and w[23] == full.nIter + 1     # restoreInfo bounds
    nri = (full.nIter + 2 - full.first) * 10
    ri = np.frombuffer(raw[4 * 24:4 * (24 + nri)], dtype="<i4").reshape(-1, 10)
    assert not ri[-1].any()                                    # entry nIter+1 never filled
    assert ri[-2, 7] == 0 and ri[-2, 8] == 0                   # no d-dagger at the last iteration
    for x, it in enumerate(range(full.first, full.nIter + 1)):
        r = full.restore[it]
        assert ri[x, 1] == r["numberOfBasis_full"] and ri[x, 9] == r["numberOfBasis"]
        assert ri[x, 3] == r["eigenvector"].size and ri[x, 5] == len(r["subspaceInfo"])
        if x:
            assert ri[x, 0] == ri[x - 1, 0] + ri[x - 1, 1] and ri[x, 2] == ri[x - 1, 2] + ri[x - 1, 3]
    # total size: header, restoreInfo, three record arrays, seven real arrays and the map
    rs, rsf = full.nVar + 3, full.nVar + 6
    nsi = sum(len(r["subspaceInfo"]) for r in full.restore.values())
    nrec = sum(r["numberOfBasis_full"] for r in full.restore.values())
    nims = sum(r["numberOfBasis"] ** 2 * full.nMat for it, r in full.restore.items() if it < full.nIter)
    nv = sum(r["eigenvector"].size for r in full.restore.values())
    # words: header 24, restoreInfo, 3 record-array sizes + records, the d-dagger size, the
    # initial d-dagger's 3 dims, 4 sizes (eigenvalues, eigenvectors, density, full
    # subspaces) + records, the map's bounds + map, 2 bin sizes
    ints = 24 + nri + 3 + (nsi + 2 * nrec) * rs + 1 + 3 + 4 + len(full.FSI) * rsf + 2 + (full.nIter + 2) + 2
    reals = nims + full.ims_initial.size + nrec + nv + full.rdm.size + 2 * full.binPos.size
    assert len(raw) == 4 * ints + 8 * reals


def test_broken_file_is_refused(case, tmp_path):
    d, full = case
    path = tmp_path / "bad.dat"
    O.run_with_restart(d, save_path=str(path), stop_before=full.startTrancation)
    raw = bytearray(path.read_bytes())
    raw[0:4] = np.array([1001], dtype="<i4").tobytes()        # MODE_RESTART_NRG
    path.write_bytes(bytes(raw))
    with pytest.raises(ValueError):
        O.load_restart(O.State(d), str(path))
