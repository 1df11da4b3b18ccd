"""CPU tests of the oracle itself (test infrastructure): an exact known answer and the
identities the reference's own runtime self-checks rely on.

The reference ships no golden vectors, so the oracle is pinned by:
* the non-interacting impurity (U = 0) without truncation: the many-body NRG spectrum of
  the last iteration and its T = 0 spectral weights must equal those built from the
  single-particle eigenstates of the same finite Wilson chain;
* spectral sum rule (1 per matrix type), RDM trace = 1 per backward step
  (reducedDensityMatrixDGEMM.F90:303-305), binned-vs-raw sums
  (calculateSpectrumDGEMM.F90:559-596);
* the loop-form legacy routines of the reference (oracle/legacy_loops.py).
"""
import itertools
import math

import numpy as np
import pytest

from oracle import nrg_oracle as O
from nrg_b200 import model

from helpers import small_siam, write_case


def _free_chain(inp, n_sites):
    """Single-particle Hamiltonian (physical units) of impurity + Wilson sites 0..n_sites-1."""
    cd, cn, _ = inp.rescaled_chains()
    first = inp.indexOfFirstIteration
    L = inp.Lambda
    h = np.zeros((n_sites + 1, n_sites + 1))
    # impurity level: eigenvalue of |up> relative to |0>, unscaled
    e_up = (inp.eigenvalue[1] - inp.eigenvalue[0]) * inp.scale(first - 1)
    h[0, 0] = e_up
    V = inp.chain_nondiagonal_raw[0, 0] * inp.scale(first)
    h[0, 1] = h[1, 0] = V
    for n in range(n_sites - 1):
        t = inp.chain_nondiagonal_raw[n - first, 0]   # physical t_n between sites n, n+1
        h[n + 1, n + 2] = h[n + 2, n + 1] = t
    return h


def test_known_answer_noninteracting_impurity(tmp_path):
    # U = 0, eps_d = 0: 5 NRG iterations -> impurity + Wilson sites 0..4, 4^6 = 4096 states
    inp = model.siam(U=0.0, Gamma=0.05, eps_d=0.0, Lambda=2.5, n_keep=100000, n_iterations=5)
    d = write_case(inp, str(tmp_path))
    st = O.run(d, spectrum=False)
    last = st.nIter
    sc = st.scale(last)
    n_sites = last - st.first + 1
    h = _free_chain(inp, n_sites)
    eps, phi = np.linalg.eigh(h)
    # many-body spectrum of free fermions, two spins, relative to the ground state
    levels = np.sort(np.concatenate([eps, eps]))
    e_mb = []
    for occ in itertools.product((0, 1), repeat=len(levels)):
        e_mb.append(float(np.dot(occ, levels)))
    e_mb = np.sort(np.array(e_mb))
    e_mb = (e_mb - e_mb[0]) / sc
    e_nrg = np.sort(st.eigenvalue)
    assert e_nrg.size == e_mb.size == 4 ** (n_sites + 1)
    assert np.max(np.abs(e_nrg - e_mb)) < 1e-10 * max(1.0, e_mb[-1])
    # T = 0 spectral weights: positive energies eps_k > 0 with |phi_k(d)|^2, per spin
    O.spike_zero_temperature(st, last)
    nbin = st.numberOfBin
    exp_pos = np.zeros((nbin * st.nMat, 2), order="F")
    exp_neg = np.zeros((nbin * st.nMat, 2), order="F")
    w = phi[0, :] ** 2
    for m in range(st.nMat):
        pos = eps > 0
        O.bin_spikes(st, exp_pos, eps[pos].copy(), w[pos].copy(), m)
        O.bin_spikes(st, exp_neg, -np.abs(eps[~pos]).copy(), w[~pos].copy(), m)
    # the two-bin split moves by ~1e3/ln(10) * dE/E per unit weight: 1e-14 relative energy
    # differences show up at ~1e-11 in individual bins
    assert np.max(np.abs(st.binPos[:, 1] - exp_pos[:, 1])) < 1e-10
    assert np.max(np.abs(st.binNeg[:, 1] - exp_neg[:, 1])) < 1e-10


@pytest.fixture(scope="module")
def truncated_run(tmp_path_factory):
    inp = small_siam(n_keep=48, n_iterations=14)
    d = write_case(inp, str(tmp_path_factory.mktemp("oracle")))
    return O.run(d)


def test_sum_rule_and_traces(truncated_run):
    st = truncated_run
    assert st.flag_truncation and st.startTrancation > st.first
    nbin = st.numberOfBin
    for m in range(st.nMat):
        tot = st.binPos[m * nbin:(m + 1) * nbin, 1].sum() + st.binNeg[m * nbin:(m + 1) * nbin, 1].sum()
        assert abs(tot - 1.0) < 1e-12
    assert st.rdm_trace, "no backward step ran"
    for N, tr in st.rdm_trace.items():
        assert abs(tr - 1.0) < 1e-12, (N, tr)
    assert not st.sum_warnings


def test_particle_hole_symmetry(truncated_run):
    # eps_d = -U/2 on a flat band: A_up(w) = A_up(-w) bin by bin
    st = truncated_run
    nbin = st.numberOfBin
    for m in range(st.nMat):
        p = st.binPos[m * nbin:(m + 1) * nbin, 1]
        q = st.binNeg[m * nbin:(m + 1) * nbin, 1]
        assert np.max(np.abs(p - q)) < 1e-9


def test_truncation_rule_keeps_whole_multiplets(truncated_run):
    st = truncated_run
    for it, flow in st.flow.items():
        if it in (st.first, st.nIter) or st.kept[it] == len(flow) and st.kept[it] <= st.truncation:
            continue
        assert st.kept[it] <= int(st.truncation * 1.2)


def test_exchange_sort_matches_reference_semantics():
    # unique keys: any correct sort; ties: the exact exchange sequence (module.F90:531-602)
    rng = np.random.default_rng(5)
    rec = np.zeros((40, 5), dtype=np.int32)
    rec[:, 0] = rng.integers(-2, 3, 40)
    rec[:, 1] = rng.integers(-2, 3, 40)
    rec[:, 2] = rng.integers(1, 6, 40)
    rec[:, 3] = np.arange(40)
    rec[:, 4] = np.arange(40)
    ref = rec.copy()
    n = len(ref)
    for i in range(n):             # the reference loop, element by element
        for j in range(i + 1, n):
            a, b = ref[i], ref[j]
            gt = (tuple(a[:2]) > tuple(b[:2])) or (tuple(a[:2]) == tuple(b[:2]) and a[2] > b[2])
            if gt:
                ref[[i, j]] = ref[[j, i]]
    out = O.exchange_sort(rec.copy(), 2)
    assert np.array_equal(out, ref)


def test_log_gaussian_broadening_keeps_the_weight():
    # one spike of weight 0.7 at E = 2e-4 (and one of weight 0.3 at -5e-3 in the negative
    # bins): the broadened curve integrates back to the weight (log grid, trapezoid in ln w)
    nbin = 5
    pos = np.zeros((nbin, 2))
    pos[:, 0] = [1e-6, 1e-5, 2e-4, 1e-3, 1e-2]
    pos[2, 1] = 0.7
    neg = np.zeros((nbin, 2))
    neg[:, 0] = -pos[:, 0]
    neg[4, 1] = 0.3
    w = O.log_grid(1e-9, 1e2, 400)
    Ap = O.broaden_log_gaussian(pos, nbin, 1, 0.6, w)[0]
    An = O.broaden_log_gaussian(neg, nbin, 1, 0.6, -w)[0]
    lnw = np.log(w)
    assert abs(np.trapezoid(Ap * w, lnw) - 0.7) <= 1e-6
    assert abs(np.trapezoid(An * w, lnw) - 0.3) <= 1e-6
    assert np.all(O.broaden_log_gaussian(pos, nbin, 1, 0.6, -w) == 0.0)
    # A(w) peaks at E, and w A(w) (the density in ln w) at E exp(b^2/2)
    assert abs(w[np.argmax(Ap)] / 2e-4 - 1.0) < 0.01
    assert abs(w[np.argmax(Ap * w)] / (2e-4 * np.exp(0.18)) - 1.0) < 0.01


def test_fdm_zero_temperature_limit_is_the_cfs_spectrum(truncated_run):
    # FDM at T << the last shell's scale: only the ground states of the last iteration
    # carry weight, and the bins are the reference-semantics CFS bins
    st = truncated_run
    bp, bn, diag = O.fdm_spectrum(st, 1e-3 * st.scale(st.nIter))
    assert np.max(np.abs(bp[:, 1] - st.binPos[:, 1])) <= 1e-8
    assert np.max(np.abs(bn[:, 1] - st.binNeg[:, 1])) <= 1e-8
    assert max(abs(t - 1.0) for t in diag["traces"].values()) <= 1e-12


@pytest.mark.parametrize("factor", [0.1, 1.0, 30.0])
def test_fdm_sum_rule_and_traces_at_finite_temperature(truncated_run, factor):
    st = truncated_run
    bp, bn, diag = O.fdm_spectrum(st, factor * st.scale(st.nIter))
    nbin = st.numberOfBin
    for m in range(st.nMat):
        tot = bp[m * nbin:(m + 1) * nbin, 1].sum() + bn[m * nbin:(m + 1) * nbin, 1].sum()
        assert abs(tot - 1.0) <= 1e-12
    assert max(abs(t - 1.0) for t in diag["traces"].values()) <= 1e-12


def test_fdm_known_answer_noninteracting_at_finite_temperature(tmp_path):
    # U = 0 without truncation: the single-particle spectral function does not depend on
    # T, so the FDM bins at any T equal |phi_k(d)|^2 at eps_k (positive or negative)
    inp = model.siam(U=0.0, Gamma=0.05, eps_d=0.0, Lambda=2.5, n_keep=100000, n_iterations=5)
    d = write_case(inp, str(tmp_path))
    st = O.run(d, spectrum=False)
    st.startTrancation = st.nIter          # one shell: the last, every state discarded
    n_sites = st.nIter - st.first + 1
    eps, phi = np.linalg.eigh(_free_chain(inp, n_sites))
    nbin = st.numberOfBin
    exp_pos = np.zeros((nbin * st.nMat, 2), order="F")
    exp_neg = np.zeros((nbin * st.nMat, 2), order="F")
    w = phi[0, :] ** 2
    for m in range(st.nMat):
        pos = eps > 0
        O.bin_spikes(st, exp_pos, eps[pos].copy(), w[pos].copy(), m)
        O.bin_spikes(st, exp_neg, -np.abs(eps[~pos]).copy(), w[~pos].copy(), m)
    for factor in (0.3, 3.0):
        bp, bn, _ = O.fdm_spectrum(st, factor * st.scale(st.nIter))
        assert np.max(np.abs(bp[:, 1] - exp_pos[:, 1])) < 1e-10
        assert np.max(np.abs(bn[:, 1] - exp_neg[:, 1])) < 1e-10
