"""The accuracy side of the precision form that the library does not build (its design
notes give the measured reasons: the plain form's time is the sequential depth of the
Householder reduction, which an FP32 reduction shares).  This CPU check keeps the
accuracy claim reproducible: eigenpairs of real NRG sector Hamiltonians computed in FP32
and refined in FP64 by Ogita and Aishima's iteration (Japan J. Indust. Appl. Math. 35,
1007-1035 (2018)) reach the FP64 eigenvalue tolerance of the parity tests (1e-12
relative) in two steps, where FP32 alone misses it by four orders of magnitude.

One step, for A symmetric and X an approximate eigenvector matrix:
R = I - X^T X, S = X^T A X, lambda_i = S_ii / (1 - R_ii); E_ij = (S_ij + lambda_j R_ij) /
(lambda_j - lambda_i) where |lambda_j - lambda_i| > delta = 2 (||S - diag(lambda)|| +
||A|| ||R||), else R_ij / 2; X <- X + X E.
"""
import numpy as np

from oracle import nrg_oracle as O
from nrg_b200 import model

from helpers import write_case


def refine(A, X):
    n = A.shape[0]
    R = np.eye(n) - X.T @ X
    S = X.T @ (A @ X)
    lam = np.diag(S) / (1.0 - np.diag(R))
    delta = 2.0 * (np.linalg.norm(S - np.diag(lam), 2) + np.linalg.norm(A, 2) * np.linalg.norm(R, 2))
    diff = lam[None, :] - lam[:, None]
    far = np.abs(diff) > delta
    E = np.where(far, (S + lam[None, :] * R) / np.where(far, diff, 1.0), R / 2.0)
    return X + X @ E, lam


def test_fp32_eigenpairs_refined_to_fp64_accuracy(tmp_path):
    inp = model.config(1, n_iterations=8)        # the N_keep = 512 workload's chain, cut after 8 iterations
    st = O.State(write_case(inp, str(tmp_path)))
    tables = (O.diag_coef_table(st), O.bcs_table(st))
    for it in range(st.first, st.nIter):
        O.nrg_iteration(st, it)
    O.prepare_basis(st, st.nIter)
    dims = st.subspaceInfo[:, st.nVar]
    checked = 0
    for s in np.argsort(-dims, kind="stable")[:4]:   # the largest sectors (order 178)
        H = O.assemble_block(st, st.nIter, int(s), tables)
        w64 = np.linalg.eigvalsh(H)
        scale = np.maximum(1.0, np.abs(w64))
        w32, U32 = np.linalg.eigh(H.astype(np.float32))
        assert np.max(np.abs(w32.astype(np.float64) - w64) / scale) > 1e-9     # FP32 alone misses 1e-12
        X = U32.astype(np.float64)
        for _ in range(2):
            X, lam = refine(H, X)
        order = np.argsort(lam)
        lam, X = lam[order], X[:, order]
        assert np.max(np.abs(lam - w64) / scale) <= 1e-12
        assert np.max(np.abs(X.T @ X - np.eye(len(H)))) <= 1e-9
        assert np.max(np.abs(H @ X - X * lam)) <= 1e-10 * np.max(np.abs(w64))
        checked += 1
    assert checked == 4 and dims.max() > 150
