"""The two rules the device-side bookkeeping of the device-resident run rests on, checked
against the oracle on the CPU (the CUDA kernels themselves are compared with the host
bookkeeping, table for table, in tests/test_gpu_tables.py):

* truncation without a sort: postprocess.F90:79-126 keeps exactly the states with
  E <= Ecut_final, where Ecut_final follows from two order statistics (the N_keep-th and
  the (limit+1)-th smallest energy) and the reference's own sequence of Ecut values;
* prepareBasis from sector-level data: after the first iteration, when the operations
  change the quantum numbers in pairwise different ways, the sorted basis and the sector
  table of prepareBasis.F90:31-114 are the (old sector, operation) runs ordered by
  (new quantum numbers, old sector).
"""
import types

import numpy as np
import pytest

from oracle import nrg_oracle as O
from nrg_b200 import model

from helpers import small_siam, write_case

THR, STEP, SCALE = 0.000001, 0.001, 1.2


def kept_by_threshold(E, n_keep, truncate):
    """The kept mask of the order-statistic form (the rule k_truncate implements)."""
    if not truncate:
        return np.ones(len(E), dtype=bool)
    limit = int(n_keep * SCALE)
    Es = np.sort(E)                      # order statistics only
    ecut = Es[n_keep - 1] + THR
    if len(E) > limit:
        el = Es[limit]                   # the (limit+1)-th smallest
        while el <= ecut:
            ecut = ecut - STEP
    return E <= ecut


def _oracle_truncate(it, first, nIter, n_keep, E):
    ns = types.SimpleNamespace(nb=len(E), eigenvalue=E.copy(), basis_output=np.zeros((len(E), 5), np.int32),
                               first=first, nIter=nIter, truncation=n_keep, startTrancation=nIter + 1,
                               flag_truncation=False, flow={}, kept={})
    O.truncate(ns, it)
    return ns


@pytest.mark.parametrize("seed", range(12))
def test_threshold_form_equals_the_sorted_rule(seed):
    rng = np.random.default_rng(100 + seed)
    nb, n_keep = 1500, 120
    E = np.round(rng.uniform(0.0, 3.0, nb), 1 + seed % 3)   # degenerate levels
    if seed % 2:      # a cluster inside the 1e-6 window wider than 1.2 N_keep: the cut-back runs
        E[rng.choice(nb, 400, replace=False)] = 0.07 + rng.uniform(0.0, 5e-7, 400)
    E[rng.integers(nb)] = 0.0
    ns = _oracle_truncate(3, -1, 20, n_keep, E)
    mask = kept_by_threshold(E, n_keep, True)
    assert int(mask.sum()) == ns.nb
    if seed % 2:
        assert ns.nb < n_keep                            # the cut-back dropped the whole cluster
    assert np.array_equal(np.flatnonzero(mask), np.sort(ns.eigenindex[:ns.nb]))


@pytest.mark.parametrize("case", ["siam", "siam_bath"])
def test_both_rules_on_every_iteration_of_a_run(case, tmp_path):
    if case == "siam":
        inp = small_siam(n_keep=64, n_iterations=16)
    else:
        inp = model.siam_bath(U=0.2, eps_d=-0.07, hybridization=lambda e: 0.02 * (1.0 + 0.4 * e), Lambda=2.5,
                              n_keep=64, n_iterations=14)
    st = O.State(write_case(inp, str(tmp_path)))
    nVar, nOps = st.nVar, st.nOps
    ops = st.operation[:, :nVar]
    assert len({tuple(r) for r in ops}) == nOps          # pairwise different changes
    prev = None                                          # (qn per sector, kept per sector)
    truncated = 0
    for it in range(st.first, st.nIter + 1):
        O.prepare_basis(st, it)
        si, bi = st.subspaceInfo, st.basis_input
        if prev is not None:
            qn_prev, kept_prev = prev
            koff = np.concatenate([[0], np.cumsum(kept_prev)])
            pairs = [(tuple(qn_prev[s] - ops[a]), s, a) for s in range(len(kept_prev)) if kept_prev[s] > 0
                     for a in range(nOps)]
            pairs.sort(key=lambda p: (p[0], p[1]))
            rows, sectors = [], []
            for q, s, a in pairs:
                if not sectors or sectors[-1][0] != q:
                    sectors.append([q, 0, len(rows)])
                sectors[-1][1] += kept_prev[s]
                rows += [(koff[s] + t + 1, t + 1, a + 1) for t in range(kept_prev[s])]
            assert np.array_equal(np.array(rows), bi[:, nVar:]), it
            ce = 1
            for k, (q, d, r0) in enumerate(sectors):
                assert tuple(si[k, :nVar]) == q and si[k, nVar] == d and si[k, nVar + 2] == r0 + 1
                assert si[k, nVar + 1] == ce
                ce += d * d
            assert len(sectors) == si.shape[0]
        O.diagonalization(st, it)
        E = st.eigenvalue.copy()
        # within a sector the eigenvalues ascend, so the kept states are the lowest columns
        for k in range(si.shape[0]):
            r0, d = si[k, nVar + 2] - 1, si[k, nVar]
            assert np.all(np.diff(E[r0:r0 + d]) >= 0)
        trunc = it != st.first and it != st.nIter and len(E) > st.truncation
        mask = kept_by_threshold(E, st.truncation, trunc)
        O.postprocess(st, it)
        assert int(mask.sum()) == st.nb, it
        truncated += st.nb < len(E)
        kept = np.array([int(mask[si[k, nVar + 2] - 1: si[k, nVar + 2] - 1 + si[k, nVar]].sum())
                         for k in range(si.shape[0])])
        prev = (si[:, :nVar].copy(), kept)
        # and the kept records are (sector qn, column 1..kept), in sector order
        exp = np.concatenate([np.column_stack([np.repeat(si[k:k + 1, :nVar], kept[k], 0),
                                               np.arange(1, kept[k] + 1)]) for k in range(si.shape[0])])
        assert np.array_equal(st.basis_output[:st.nb, :nVar + 1], exp), it
    assert truncated > 0
