"""nrg_block_eigh_noalloc: the eigensolver entry point that allocates no device memory.

It serves callers that cannot allocate on the device (their pool allocator owns the GPU,
or they must not trigger cudaMalloc's implicit synchronisation mid-stream).  This test
calls it through the C ABI on device arrays the test owns, twice in a row (the static
workspace keeps the previous call's contents), and checks each result against the
existing entry point nrg_diagonalization on the same sector Hamiltonian, within the
tolerances of the other parity tests (eigenvalues 1e-12 relative, eigenvector
projectors 1e-9).  This file is collected last so a failure here comes after every other
test has run.
"""
import ctypes

import numpy as np
import pytest

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


def test_block_eigh_noalloc_matches_diagonalization(ctx_factory):
    torch = pytest.importorskip("torch")
    lib = load_library()
    fn = lib.nrg_block_eigh_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    cases = _sectors(ctx_factory)
    assert len(cases) == 2
    dev = torch.device("cuda", 0)
    for H, E_ref, V_ref in cases:            # two calls in a row, different orders
        n = H.shape[0]
        dH = torch.tensor(np.asfortranarray(H).ravel(order="F"), dtype=torch.float64, device=dev)
        dw = torch.zeros(n, dtype=torch.float64, device=dev)
        dV = torch.zeros(n * n, dtype=torch.float64, device=dev)
        rc = fn(dH.data_ptr(), n, dw.data_ptr(), dV.data_ptr(), None)
        assert rc == 0, lib.nrg_last_error()
        w = dw.cpu().numpy()
        V = dV.cpu().numpy().reshape((n, n), order="F")
        V[np.abs(V) < 1e-14] = 0.0       # nrg_diagonalization chops (diagonalization.F90:392-399)
        assert eig_rel_err(w, E_ref) <= 1e-12
        assert subspace_err(V, V_ref, w) <= 1e-9
        assert np.allclose(H @ V, V * w, atol=1e-12 * max(1.0, np.max(np.abs(w))))
    # orders beyond the static workspace are rejected without touching the device arrays
    rc = fn(dH.data_ptr(), MAX_ORDER + 1, dw.data_ptr(), dV.data_ptr(), None)
    assert rc == 4
