"""Wilson chains for an arbitrary hybridisation function (the input side of a run).

The reference reads its chain from ``initial.dat`` (read_initial_basis.F90:27-204), made
by a generator that is not part of it.  This module makes the chain for a bath given by
its hybridisation function Gamma(eps) = pi sum_k |V_k|^2 delta(eps - eps_k) on [-D, D]:

1. logarithmic discretisation: intervals D Lambda^{-(m+z-1)} .. D Lambda^{-(m+z)} on each
   side (m = 0, 1, ...; the first interval of a side starts at D), each replaced by one
   bath level of weight gamma_m^2 = (1/pi) int_I Gamma and energy
   * "wilson": the mean int_I Gamma eps / int_I Gamma (Wilson, Rev. Mod. Phys. 47, 773
     (1975)); for a flat band this is eq. (2.15) and wants the A_Lambda correction of the
     coupling;
   * "campo": int_I Gamma / int_I Gamma/eps (Campo and Oliveira, Phys. Rev. B 72, 104432
     (2005)), which removes most of the discretisation error without a correction;
2. the star (bath levels coupled to the impurity) to chain map: the chain's on-site
   energies eps_n and hoppings t_n are the recurrence coefficients of the polynomials
   orthogonal on the discrete measure {xi_m, gamma_m^2}, computed by Lanczos in decimal
   arithmetic with enough digits for the Lambda^{-n/2} decay of the coefficients;
   V = sqrt(sum gamma_m^2) couples the impurity to site 0.

Energies are in the units of D; the outputs are the physical (unrescaled) values that
initial.dat holds.
"""
from __future__ import annotations

import decimal
import math
from typing import Callable, Tuple

import numpy as np
import scipy.integrate


def _interval_integrals(gamma: Callable[[float], float], a: float, b: float, scheme: str):
    """(int Gamma, representative energy) on [a, b] with 0 <= a < b (positive side)."""
    opts = dict(limit=200, epsabs=0.0, epsrel=1e-13)
    w = scipy.integrate.quad(gamma, a, b, **opts)[0]
    if w <= 0.0:
        return 0.0, 0.0
    if scheme == "wilson":
        e = scipy.integrate.quad(lambda x: gamma(x) * x, a, b, **opts)[0] / w
    elif scheme == "campo":
        e = w / scipy.integrate.quad(lambda x: gamma(x) / x, a, b, **opts)[0]
    else:
        raise ValueError("scheme must be 'wilson' or 'campo'")
    return w, e


def star(gamma: Callable[[float], float], D: float, Lambda: float, n_intervals: int, z: float = 1.0,
         scheme: str = "campo") -> Tuple[np.ndarray, np.ndarray]:
    """Bath levels (energies xi, weights gamma^2) of the logarithmic discretisation, both
    sides, ``n_intervals`` per side; the remainder next to the Fermi level (weight of
    order Lambda^-n_intervals) is left out."""
    if Lambda <= 1.0 or D <= 0.0 or n_intervals < 1 or not 0.0 < z <= 1.0:
        raise ValueError("need Lambda > 1, D > 0, n_intervals >= 1, 0 < z <= 1")
    edges = [D] + [D * Lambda ** (-(m + z)) for m in range(n_intervals)]
    xi, w = [], []
    for sign in (1.0, -1.0):
        g = (lambda x, s=sign: max(0.0, float(gamma(s * x))))
        for m in range(n_intervals):
            a, b = edges[m + 1], edges[m]
            wt, e = _interval_integrals(g, a, b, scheme)
            if wt > 0.0:
                xi.append(sign * e)
                w.append(wt / math.pi)
    return np.array(xi), np.array(w)


def star_to_chain(xi, w, n_sites: int, digits: int = 0) -> Tuple[float, np.ndarray, np.ndarray]:
    """Chain (V, eps[0:n_sites], t[0:n_sites-1]) of the star {xi, w}: H = sum_n eps_n
    f_n^dag f_n + sum_n t_n (f_n^dag f_{n+1} + h.c.), V^2 = sum w, site 0 the bath
    orbital the impurity couples to.

    Lanczos on diag(xi) from the start vector sqrt(w)/V with full reorthogonalisation, in
    ``digits``-digit decimal arithmetic.  The Lanczos vectors stay normalised, so the
    absolute error of a coefficient is ~10^-digits and its relative error
    10^-digits Lambda^{n/2}: the default takes 30 digits beyond the coefficients' decay.
    (The equivalent recurrence on orthogonal polynomials needs digits quadratic in n.)"""
    xi = [float(x) for x in xi]
    w = [float(x) for x in w]
    if len(xi) != len(w) or not w or min(w) < 0.0:
        raise ValueError("star energies and non-negative weights of equal length needed")
    if n_sites > len(xi):
        raise ValueError(f"{len(xi)} bath levels give at most {len(xi)} chain sites")
    eps = np.zeros(n_sites)
    t = np.zeros(max(n_sites - 1, 0))
    with decimal.localcontext() as ctx:     # every operator below works at this precision
        ctx.prec = digits if digits > 0 else 30
        X = [decimal.Decimal(x) for x in xi]   # exact binary values of the doubles
        W = [decimal.Decimal(x) for x in w]
        zero = decimal.Decimal(0)
        norm0 = sum(W, zero).sqrt()
        basis = []
        beta = zero
        u = [wk.sqrt() / norm0 for wk in W]
        for n in range(n_sites):
            a = sum((xk * uk * uk for xk, uk in zip(X, u)), zero)
            eps[n] = float(a)
            if n == n_sites - 1:
                break
            r = [xk * uk - a * uk for xk, uk in zip(X, u)]
            if basis:
                r = [rk - beta * pk for rk, pk in zip(r, basis[-1])]
            basis.append(u)
            for _ in range(2):   # full reorthogonalisation, twice
                for v in basis:
                    c = sum((rk * vk for rk, vk in zip(r, v)), zero)
                    r = [rk - c * vk for rk, vk in zip(r, v)]
            beta = sum((rk * rk for rk in r), zero).sqrt()
            if beta == 0:
                raise ValueError(f"the star ends the chain at site {n + 1}")
            t[n] = float(beta)
            if digits <= 0:   # keep 30 digits below the current coefficient
                ctx.prec = max(ctx.prec, 30 + int(max(0.0, -math.log10(float(beta)))) + 1)
            u = [rk / beta for rk in r]
        v = float(norm0)
    return v, eps, t


def log_discretized_chain(gamma: Callable[[float], float], D: float, Lambda: float, n_sites: int,
                          z: float = 1.0, scheme: str = "campo", extra_intervals: int = 0
                          ) -> Tuple[float, np.ndarray, np.ndarray]:
    """(V, eps, t) of the Wilson chain of the bath with hybridisation function ``gamma``
    on [-D, D]: ``n_sites`` on-site energies and ``n_sites - 1`` hoppings.

    Each side is cut into n_sites/2 + ``extra_intervals`` intervals.  The levels left out
    next to the Fermi level (weight ~Lambda^-M for M intervals) change coefficient n by
    ~Lambda^{n/2-M} relative, so the default extra count, 15/log10(Lambda) + 4, keeps
    that below 1e-15."""
    if extra_intervals <= 0:
        extra_intervals = int(math.ceil(15.0 / math.log10(Lambda))) + 4
    xi, w = star(gamma, D, Lambda, n_sites // 2 + extra_intervals, z, scheme)
    return star_to_chain(xi, w, n_sites)
