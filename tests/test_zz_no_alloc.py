"""nrg_block_eigh_noalloc: the eigensolver entry point that allocates no device memory.

It serves callers that cannot allocate on the device (their pool allocator owns the GPU,
or they must not trigger cudaMalloc's implicit synchronisation mid-stream).  This test
calls it through the C ABI on device arrays the test owns, twice in a row (the static
workspace keeps the previous call's contents), and checks each result against the
existing entry point nrg_diagonalization on the same sector Hamiltonian, within the
tolerances of the other parity tests (eigenvalues 1e-12 relative, eigenvector
projectors 1e-9), and with the oracle's LAPACK dsyev on the same blocks.  A second test
covers the edges: orders 1 and the static limit, the in-place call, a block holding NaN,
orders beyond the limit and host arrays (rejected), and that repeated calls leave the
device's free memory unchanged.  This file is collected last so a failure here comes after
every other test has run.
"""
import ctypes

import numpy as np
import pytest
import scipy.linalg

from oracle import nrg_oracle as O
from nrg_b200 import model, load_library

from helpers import eig_rel_err, small_siam, subspace_err, write_case, sector_blocks

pytestmark = pytest.mark.gpu

MAX_ORDER = 128


def _sectors(ctx_factory):
    inp = small_siam(n_keep=256, n_iterations=7)
    d = write_case(inp)
    st = O.State(d)
    ctx = ctx_factory(model.read_inputs(d))
    tables = (O.diag_coef_table(st), O.bcs_table(st))
    for it in range(st.first, st.nIter + 1):
        O.prepare_basis(st, it)
        si, bi = st.subspaceInfo.copy(), st.basis_input.copy()
        Eold, IMold = st.eigenvalue.copy(), st.im.copy(order="F")
        E_g, V_g, _, _ = ctx.diagonalization(it, si, bi, Eold, IMold)
        st.eigenvalue_prev, st.im_prev = st.eigenvalue, st.im
        dims = si[:, st.nVar]
        if it >= 3 and dims.max() >= 60:
            picks = []
            order = np.argsort(-dims)
            for s in order:
                if dims[s] <= MAX_ORDER and len(picks) < 2:
                    picks.append(int(s))
            out = []
            # the existing entry point shifted all eigenvalues by the global minimum
            shift = float(np.min(np.concatenate([np.linalg.eigvalsh(O.assemble_block(st, it, k, tables))
                                                 for k in range(st.numberOfSubspace)])))
            blocks = {s: B for s, _, B in sector_blocks(si, V_g, st.nVar)}
            for s in picks:
                H = O.assemble_block(st, it, s, tables)
                s0 = int(si[s, st.nVar + 2]) - 1
                dd = int(dims[s])
                out.append((H, E_g[s0:s0 + dd] + shift, blocks[s]))
            return out
        O.diagonalization(st, it)
        O.postprocess(st, it)
    raise AssertionError("no suitable sector")


def _entry():
    lib = load_library()
    fn = lib.nrg_block_eigh_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return lib, fn


def _solve(fn, torch, H, in_place=False):
    """One call on device copies of H; returns (status, eigenvalues, eigenvectors)."""
    n = H.shape[0]
    dev = torch.device("cuda", 0)
    dH = torch.tensor(np.asfortranarray(H).ravel(order="F"), dtype=torch.float64, device=dev)
    dw = torch.zeros(n, dtype=torch.float64, device=dev)
    dV = dH if in_place else torch.zeros(n * n, dtype=torch.float64, device=dev)
    rc = fn(dH.data_ptr(), n, dw.data_ptr(), dV.data_ptr(), None)
    return rc, dw.cpu().numpy(), dV.cpu().numpy().reshape((n, n), order="F")


def _check(H, w, V, w_ref, V_ref):
    assert eig_rel_err(w, w_ref) <= 1e-12
    assert subspace_err(V, V_ref, w) <= 1e-9
    assert np.allclose(H @ V, V * w, atol=1e-12 * max(1.0, np.max(np.abs(w))))


def test_block_eigh_noalloc_matches_diagonalization(ctx_factory):
    torch = pytest.importorskip("torch")
    lib, fn = _entry()
    cases = _sectors(ctx_factory)
    assert len(cases) == 2
    for H, E_ref, V_ref in cases:            # two calls in a row, different orders
        rc, w, V = _solve(fn, torch, H)
        assert rc == 0, lib.nrg_last_error()
        V[np.abs(V) < 1e-14] = 0.0       # nrg_diagonalization chops (diagonalization.F90:273-280)
        _check(H, w, V, E_ref, V_ref)
        # and the oracle's dsyev('V', 'U') on the same block
        w_o, V_o = scipy.linalg.eigh(H, lower=False, driver="ev")
        _check(H, w, V, w_o, V_o)


def test_block_eigh_noalloc_edges():
    torch = pytest.importorskip("torch")
    lib, fn = _entry()
    rng = np.random.default_rng(20261204)
    for n in (1, 2, 127, MAX_ORDER):        # the one-element path, and the static limit itself
        A = rng.standard_normal((n, n))
        H = 0.5 * (A + A.T)
        w_o, V_o = np.linalg.eigh(H)
        rc, w, V = _solve(fn, torch, H)
        assert rc == 0, lib.nrg_last_error()
        _check(H, w, V, w_o, V_o)
    # in place: the eigenvectors overwrite H
    A = rng.standard_normal((96, 96))
    H = 0.5 * (A + A.T)
    rc, w, V = _solve(fn, torch, H, in_place=True)
    assert rc == 0, lib.nrg_last_error()
    w_o, V_o = np.linalg.eigh(H)
    _check(H, w, V, w_o, V_o)
    # a block with a NaN is reported, and the next call works again
    Hn = H.copy()
    Hn[3, 5] = Hn[5, 3] = np.nan
    rc, _, _ = _solve(fn, torch, Hn)
    assert rc == 8, lib.nrg_last_error()                # NRG_ERR_NUMERIC
    rc, w, V = _solve(fn, torch, H)
    assert rc == 0, lib.nrg_last_error()
    _check(H, w, V, w_o, V_o)
    # orders beyond the static workspace, and host arrays, are rejected without a launch
    dev = torch.device("cuda", 0)
    d = torch.zeros((MAX_ORDER + 1) ** 2, dtype=torch.float64, device=dev)
    assert fn(d.data_ptr(), MAX_ORDER + 1, d.data_ptr(), d.data_ptr(), None) == 4   # NRG_ERR_TOO_LARGE
    h = np.zeros(16)
    assert fn(h.ctypes.data, 4, d.data_ptr(), d.data_ptr(), None) == 1              # NRG_ERR_INVALID
    # the call allocates nothing: the device's free memory is the same after two more calls
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(0)[0]
    dH = torch.tensor(np.asfortranarray(H).ravel(order="F"), dtype=torch.float64, device=dev)
    dw = torch.zeros(96, dtype=torch.float64, device=dev)
    dV = torch.zeros(96 * 96, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info(0)[0]
    for _ in range(2):
        assert fn(dH.data_ptr(), 96, dw.data_ptr(), dV.data_ptr(), None) == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(0)[0] == free1, (free0, free1)
