"""Shared test helpers: input directories and comparisons that respect eigenvector gauge."""
import os
import tempfile

import numpy as np

from nrg_b200 import model


def write_case(inp, root=None):
    d = tempfile.mkdtemp(prefix="nrg_case_", dir=root)
    model.write_inputs(inp, d)
    return d


def small_siam(n_keep=48, n_iterations=14, **kw):
    args = dict(U=0.1, Gamma=0.01, eps_d=-0.05, Lambda=2.5, n_keep=n_keep, n_iterations=n_iterations)
    args.update(kw)
    return model.siam(**args)


def eig_rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b) / np.maximum(1.0, np.abs(b)))) if a.size else 0.0


def subspace_err(Va, Vb, E, cluster_tol=1e-5):
    """Largest projector difference over clusters of (near-)degenerate eigenvalues.

    Columns of Va and Vb are eigenvectors sorted by the ascending eigenvalues E; each
    cluster's eigenvectors are determined only up to a rotation, so compare projectors.
    Eigenvectors of a backward-stable solver move by ~eps*|H|/gap, so eigenvalues closer
    than cluster_tol (relative) are grouped: outside the groups that bound is ~2e-10.
    """
    n = len(E)
    worst = 0.0
    i = 0
    while i < n:
        j = i + 1
        while j < n and E[j] - E[j - 1] <= cluster_tol * max(1.0, abs(E[j])):
            j += 1
        Pa = Va[:, i:j] @ Va[:, i:j].T
        Pb = Vb[:, i:j] @ Vb[:, i:j].T
        worst = max(worst, float(np.max(np.abs(Pa - Pb))))
        i = j
    return worst


def sector_blocks(si, V, nVar):
    """Yield (isub, d, block) for the column-major eigenvector blocks of one iteration."""
    for s in range(si.shape[0]):
        d = int(si[s, nVar])
        c0 = int(si[s, nVar + 1]) - 1
        yield s, d, V[c0:c0 + d * d].reshape((d, d), order="F")
