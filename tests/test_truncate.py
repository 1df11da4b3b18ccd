"""postprocess's truncation and reorder through the C ABI (nrg_truncate) against the
oracle, bit for bit, on the CPU (postprocess.F90:69-168): the stable energy sort, the
kept count (N_keep extended over the 1e-6 window, cut back by 0.001 steps to at most
1.2 N_keep), the kept states in index order followed by the discarded ones in energy
order, and the first truncated iteration."""
import types

import numpy as np
import pytest

from oracle import nrg_oracle as O
from nrg_b200 import model, truncate

from helpers import small_siam, write_case


@pytest.mark.parametrize("case", ["siam", "two_orbital"])
def test_every_iteration_of_a_run_matches_the_oracle(case, tmp_path):
    inp = (small_siam(n_keep=48, n_iterations=14) if case == "siam"
           else model.two_orbital_hund(n_keep=96, n_iterations=5))
    st = O.State(write_case(inp, str(tmp_path)))
    truncated = 0
    for it in range(st.first, st.nIter + 1):
        O.prepare_basis(st, it)
        O.diagonalization(st, it)
        E, bo, kept, s_t, f_t = truncate(it, st.first, st.nIter, st.truncation, st.nVar, st.eigenvalue,
                                         st.basis_output, st.startTrancation, st.flag_truncation)
        O.postprocess(st, it)
        assert kept == st.nb, it
        assert np.array_equal(E, st.eigenvalue), it
        assert np.array_equal(bo, st.basis_output), it
        assert (s_t, f_t) == (st.startTrancation, st.flag_truncation), it
        truncated += kept < len(E)
    assert truncated > 0


def _oracle(it, first, nIter, n_keep, E, bo):
    ns = types.SimpleNamespace(nb=len(E), eigenvalue=E.copy(), basis_output=bo.copy(), first=first,
                               nIter=nIter, truncation=n_keep, startTrancation=nIter + 1,
                               flag_truncation=False, flow={}, kept={})
    O.truncate(ns, it)
    return ns


@pytest.mark.parametrize("seed", range(6))
def test_degenerate_levels_and_the_cut_back_loop(seed):
    rng = np.random.default_rng(seed)
    nb, n_keep = 1200, 100
    E = np.round(rng.uniform(0.0, 3.0, nb), 1)           # ~30 levels, each ~40-fold degenerate
    if seed % 2:
        # 300 levels within 1e-6 of E(N_keep): the window exceeds 1.2 N_keep, so the cutoff
        # is pulled back in 0.001 steps
        E[rng.choice(nb, 300, replace=False)] = 0.05 + rng.uniform(0.0, 5e-7, 300)
    E[rng.integers(nb)] = 0.0
    bo = np.zeros((nb, 5), dtype=np.int32)
    bo[:, 0] = rng.integers(-3, 4, nb)
    bo[:, 2] = np.arange(1, nb + 1)
    ns = _oracle(4, -1, 20, n_keep, E, bo)
    E2, bo2, kept, s_t, f_t = truncate(4, -1, 20, n_keep, 2, E, bo, 21, False)
    assert kept == ns.nb and 0 < kept <= int(1.2 * n_keep)
    if seed % 2:
        assert kept < n_keep                           # the cut-back dropped the whole cluster
    assert np.array_equal(E2, ns.eigenvalue) and np.array_equal(bo2, ns.basis_output)
    assert (s_t, f_t) == (4, True)


def test_no_truncation_at_the_first_and_last_iterations():
    rng = np.random.default_rng(1)
    E = rng.uniform(0.0, 1.0, 500)
    bo = np.zeros((500, 5), dtype=np.int32)
    bo[:, 2] = np.arange(1, 501)
    for it in (-1, 20):
        E2, bo2, kept, s_t, f_t = truncate(it, -1, 20, 100, 2, E, bo, 21, False)
        assert kept == 500 and np.array_equal(E2, E) and np.array_equal(bo2, bo) and (s_t, f_t) == (21, False)
