"""Failure detection without a GPU fault: bad input planted on the host.

The reference checks nothing here (dsyev's info is ignored, diagonalization.F90:267-268).
The library's assembly kernel checks every gathered index and every assembled value and
reports through the device status word instead of reading out of bounds or diagonalising
NaN: the flagged entries are stored as 0, so the eigensolver runs on a finite matrix, and
the call returns an error status.  Each case here plants the fault in a host module array
handed to nrg_diagonalization (the drop-in entry), checks the status and message, then
checks that the same context still gives the oracle's result on clean input.
"""
import numpy as np
import pytest

from oracle import nrg_oracle as O
from nrg_b200 import NrgError, model

from helpers import eig_rel_err, write_case

pytestmark = pytest.mark.gpu


def _state_at(iteration):
    # the bench workload's chain: iteration 4 has sectors above order 128 (the large-sector
    # eigensolver) and below (one block per sector)
    inp = model.config(2, n_iterations=6)
    d = write_case(inp)
    st = O.State(d)
    for it in range(st.first, iteration):
        O.nrg_iteration(st, it)
    O.prepare_basis(st, iteration)
    return d, st


def test_nonfinite_and_bad_index_are_reported(ctx_factory):
    it = 4
    d, st = _state_at(it)
    ctx = ctx_factory(model.read_inputs(d))
    si, bi = st.subspaceInfo.copy(), st.basis_input.copy()
    Eold, IMold = st.eigenvalue.copy(), st.im.copy(order="F")
    nVar, nOps = st.nVar, st.nOps
    assert int(np.max(si[:, nVar])) > 128

    # NaN in the previous eigenvalues: every diagonal entry built from that state
    E_bad = Eold.copy()
    E_bad[0] = np.nan
    with pytest.raises(NrgError) as e:
        ctx.diagonalization(it, si, bi, E_bad, IMold)
    assert e.value.status == 8 and "0x8" in str(e.value)       # NRG_ERR_NUMERIC

    # Inf in the invariant matrix the off-diagonal blocks are gathered from
    IM_bad = IMold.copy(order="F")
    IM_bad[:, :, 0] = np.inf
    with pytest.raises(NrgError) as e:
        ctx.diagonalization(it, si, bi, Eold, IM_bad)
    assert e.value.status == 8

    # a basis_input group whose references point past the previous iteration's states: the
    # host's table checks pass (consecutive references), the kernel's bounds check fires
    nbo = IMold.shape[0]
    bi_bad = bi.copy()
    s = int(np.argmax(si[:, nVar]))
    b0, dd = int(si[s, nVar + 2]) - 1, int(si[s, nVar])
    rows = [r for r in range(b0, b0 + dd) if bi[r, nVar + 2] == 1]
    assert rows
    bi_bad[rows, nVar] += nbo
    with pytest.raises(NrgError) as e:
        ctx.diagonalization(it, si, bi_bad, Eold, IMold)
    assert e.value.status == 1 and "0x1" in str(e.value)       # NRG_ERR_INVALID

    # the context is still usable: clean input gives the oracle's eigenvalues
    E_g, _, bo_g, _ = ctx.diagonalization(it, si, bi, Eold, IMold)
    O.diagonalization(st, it)
    assert np.array_equal(bo_g, st.basis_output)
    assert eig_rel_err(E_g, st.eigenvalue) <= 1e-12
    assert nOps == 4
