"""prepareBasis through the C ABI (nrg_prepare_basis) against the oracle, bit for bit, on
the CPU: the product basis, the sortBasisArray order (module.F90:531-602; an exchange
sort whose order among equal keys the two-orbital model exercises: several operations
shift the quantum numbers alike) and the sector table (prepareBasis.F90:1-119)."""
import types

import numpy as np
import pytest

from oracle import nrg_oracle as O
from nrg_b200 import model, prepare_basis

from helpers import small_siam, write_case


def _oracle(operation, nVar, bo):
    ns = types.SimpleNamespace(nVar=nVar, nOps=operation.shape[0], numberOfBasis_old=bo.shape[0],
                               basis_output=bo, operation=operation)
    O.prepare_basis(ns, 0)
    return ns.basis_input, ns.subspaceInfo


@pytest.mark.parametrize("case", ["siam", "two_orbital"])
def test_every_iteration_of_a_run_matches_the_oracle(case, tmp_path):
    inp = (small_siam(n_keep=48, n_iterations=10) if case == "siam"
           else model.two_orbital_hund(n_keep=96, n_iterations=5))
    st = O.State(write_case(inp, str(tmp_path)))
    ties = 0
    for it in range(st.first, st.nIter + 1):
        bo = np.ascontiguousarray(st.basis_output[:st.numberOfBasis_old], dtype=np.int32)
        bi, si = prepare_basis(st.operation, st.nVar, bo)
        O.prepare_basis(st, it)
        assert np.array_equal(bi, st.basis_input), it
        assert np.array_equal(si, st.subspaceInfo), it
        key = bi[:, :st.nVar + 1]
        ties += int(np.sum(np.all(key[1:] == key[:-1], axis=1)))
        O.diagonalization(st, it)
        O.postprocess(st, it)
    assert (ties > 0) == (case == "two_orbital")


def test_large_two_orbital_basis_with_ties_matches_the_oracle():
    # ~1200 kept states in sectors of the two-orbital model's quantum numbers (charge,
    # 2Sz) -> ~19,000 records, many with equal (quantum numbers, reference)
    ops = np.asarray(model.two_orbital_hund(n_keep=8, n_iterations=2).operation, dtype=np.int32)
    nVar = 2
    rng = np.random.default_rng(7)
    rows = []
    for q in range(-6, 7):
        for sz in range(-6, 7, 2):
            for v in range(1, int(rng.integers(5, 20)) + 1):
                rows.append([q, sz, v, 0, 0])
    bo = np.array(rows, dtype=np.int32)
    assert bo.shape[0] > 1000
    bi, si = prepare_basis(ops, nVar, bo)
    bi_ref, si_ref = _oracle(ops, nVar, bo)
    assert np.array_equal(bi, bi_ref) and np.array_equal(si, si_ref)
    key = bi[:, :nVar + 1]
    assert np.sum(np.all(key[1:] == key[:-1], axis=1)) > 1000


def test_rejects_inconsistent_arguments():
    from nrg_b200 import NrgError
    ops = np.zeros((4, 3), dtype=np.int32)
    with pytest.raises(NrgError):
        prepare_basis(ops, 0, np.zeros((2, 3), dtype=np.int32))
