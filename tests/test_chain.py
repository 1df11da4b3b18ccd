"""Wilson chains for an arbitrary bath (nrg_b200.chain, model.siam_bath) on the CPU.

Known answers: Wilson's flat-band hoppings (Rev. Mod. Phys. 47, 773, eq. 2.15); the
Campo-Oliveira flat-band chain, which is Wilson's divided by A_Lambda (same weights,
energies scaled by 1/A_Lambda); zero on-site energies for a particle-hole symmetric
bath; the chain of a whole star reproduces the star's levels and weights; and through
the oracle, the NRG spectrum of a non-interacting impurity on a particle-hole asymmetric
bath equals the free-fermion spectrum of the same chain, and its T = 0 spectral weights
the single-particle weights |phi_k(d)|^2 at eps_k."""
import itertools
import math

import numpy as np
import pytest
import scipy.integrate

from oracle import nrg_oracle as O
from nrg_b200 import chain, model

from helpers import write_case


@pytest.mark.parametrize("Lambda", [2.0, 2.5, 3.0])
def test_flat_band_reproduces_wilsons_hoppings(Lambda):
    V, eps, t = chain.log_discretized_chain(lambda e: 0.05, 1.0, Lambda, 62, scheme="wilson")
    tw = model.wilson_flat_band_hoppings(Lambda, 1.0, 61)
    assert np.max(np.abs(t - tw) / tw) <= 1e-12
    assert np.max(np.abs(eps[:-1]) / tw) <= 1e-20
    assert abs(V - math.sqrt(2 * 0.05 / math.pi)) <= 1e-12 * V


def test_campo_flat_band_is_wilsons_over_a_lambda():
    L = 2.5
    _, _, tw = chain.log_discretized_chain(lambda e: 0.05, 1.0, L, 50, scheme="wilson")
    _, _, tc = chain.log_discretized_chain(lambda e: 0.05, 1.0, L, 50, scheme="campo")
    a = 0.5 * (1 + 1 / L) * math.log(L) / (1 - 1 / L)
    assert np.max(np.abs(tc * a - tw) / tw) <= 1e-12


def test_symmetric_bath_has_no_on_site_energies():
    g = (lambda e: 0.04 * math.sqrt(max(0.0, 1.0 - e * e)))          # semicircular
    V, eps, t = chain.log_discretized_chain(g, 1.0, 2.0, 50)
    assert np.max(np.abs(eps[:-1]) / t) <= 1e-12
    total = scipy.integrate.quad(g, -1.0, 1.0, epsabs=0, epsrel=1e-13)[0] / math.pi
    assert abs(V * V - total) <= 1e-8 * total                        # tail left out: ~2^-40
    assert np.all(np.diff(np.log(t[10:])) < 0)                       # decaying ~Lambda^-n/2


def test_chain_of_a_whole_star_has_its_levels_and_weights():
    xi = np.array([-0.9, -0.3, -0.05, -0.01, 0.02, 0.07, 0.4, 0.8])
    w = np.array([0.1, 0.3, 0.05, 0.02, 0.04, 0.2, 0.15, 0.12])
    V, eps, t = chain.star_to_chain(xi, w, len(xi))
    H = np.diag(eps) + np.diag(t, 1) + np.diag(t, -1)
    e, v = np.linalg.eigh(H)
    assert np.max(np.abs(e - np.sort(xi))) <= 1e-13
    assert np.max(np.abs(v[0, :] ** 2 - w[np.argsort(xi)] / V ** 2)) <= 1e-13
    assert abs(V * V - w.sum()) <= 1e-15


def test_asymmetric_bath_gives_on_site_energies():
    V, eps, t = chain.log_discretized_chain(lambda e: 0.05 * (1.0 + 0.6 * e), 1.0, 2.0, 40)
    assert np.max(np.abs(eps[:10])) > 1e-3


def test_noninteracting_impurity_on_an_asymmetric_bath(tmp_path):
    # U = 0, no truncation: the NRG levels of the last iteration are the free-fermion
    # many-body levels of impurity + chain, on-site energies included
    inp = model.siam_bath(U=0.0, eps_d=0.01, hybridization=lambda e: 0.05 * (1.0 + 0.6 * e),
                          Lambda=2.5, n_keep=100000, n_iterations=5)
    assert np.any(inp.chain_diagonal_raw != 0.0)
    d = write_case(inp, str(tmp_path))
    back = model.read_inputs(d)
    assert np.array_equal(back.chain_diagonal_raw, inp.chain_diagonal_raw)
    st = O.run(d, spectrum=False)
    first, last = st.first, st.nIter
    n_sites = last - first + 1
    h = np.zeros((n_sites + 1, n_sites + 1))
    h[0, 0] = (inp.eigenvalue[1] - inp.eigenvalue[0]) * inp.scale(first - 1)     # eps_d
    h[0, 1] = h[1, 0] = inp.chain_nondiagonal_raw[0, 0] * inp.scale(first)      # V
    for n in range(n_sites):
        h[n + 1, n + 1] = inp.chain_diagonal_raw[n, 0]
        if n + 1 < n_sites:
            h[n + 1, n + 2] = h[n + 2, n + 1] = inp.chain_nondiagonal_raw[n - first, 0]
    levels = np.sort(np.concatenate([np.linalg.eigvalsh(h)] * 2))
    e_mb = np.sort([float(np.dot(occ, levels)) for occ in itertools.product((0, 1), repeat=len(levels))])
    e_mb = (e_mb - e_mb[0]) / st.scale(last)
    e_nrg = np.sort(st.eigenvalue)
    assert e_nrg.size == e_mb.size
    assert np.max(np.abs(e_nrg - e_mb)) < 1e-10 * max(1.0, e_mb[-1])
    # T = 0 spectral weights: |phi_k(d)|^2 at eps_k, positive or negative (one spin)
    O.spike_zero_temperature(st, last)
    eps, phi = np.linalg.eigh(h)
    nbin = st.numberOfBin
    exp_pos = np.zeros((nbin * st.nMat, 2), order="F")
    exp_neg = np.zeros((nbin * st.nMat, 2), order="F")
    w = phi[0, :] ** 2
    for m in range(st.nMat):
        pos = eps > 0
        O.bin_spikes(st, exp_pos, eps[pos].copy(), w[pos].copy(), m)
        O.bin_spikes(st, exp_neg, -np.abs(eps[~pos]).copy(), w[~pos].copy(), m)
    assert np.max(np.abs(st.binPos[:, 1] - exp_pos[:, 1])) < 1e-10
    assert np.max(np.abs(st.binNeg[:, 1] - exp_neg[:, 1])) < 1e-10
    assert abs(w[eps > 0].sum() - w[eps < 0].sum()) > 1e-3          # the asymmetry shows
