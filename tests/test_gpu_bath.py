"""A particle-hole asymmetric bath on the GPU (model.siam_bath): the only workload whose
Wilson chain has on-site energies (chain_diagonal, the H_ii term of
diagonalization.F90:166-171), run whole on the device and compared with the oracle.

Tolerances as in the routine parity tests: kept counts identical, bins within 1e-8
absolute, sum rule within 1e-10, lowest levels within 1e-11 relative."""
import numpy as np
import pytest

from oracle import nrg_oracle as O
from nrg_b200 import model

from helpers import write_case

pytestmark = pytest.mark.gpu


def test_asymmetric_bath_run_matches_oracle(ctx_factory):
    inp = model.siam_bath(U=0.1, eps_d=-0.03, hybridization=lambda e: 0.02 * (1.0 + 0.6 * e),
                          Lambda=2.5, n_keep=48, n_iterations=14)
    assert np.max(np.abs(inp.chain_diagonal_raw)) > 1e-4
    d = write_case(inp)
    st = O.run(d)
    ctx = ctx_factory(model.read_inputs(d))
    for host_drop_in in (False, True):
        res = ctx.run(spectrum=True, host_drop_in=host_drop_in)
        its = list(range(st.first, st.nIter + 1))
        assert [int(k) for k in res["kept"]] == [st.kept[i] for i in its]
        assert np.max(np.abs(res["binPos"][:, 1] - st.binPos[:, 1])) <= 1e-8
        assert np.max(np.abs(res["binNeg"][:, 1] - st.binNeg[:, 1])) <= 1e-8
        nbin = st.numberOfBin
        for m in range(st.nMat):
            tot = res["binPos"][m * nbin:(m + 1) * nbin, 1].sum() + res["binNeg"][m * nbin:(m + 1) * nbin, 1].sum()
            assert abs(tot - 1.0) <= 1e-10
        for k, i in enumerate(its):
            flow = st.flow[i][:8]
            assert np.max(np.abs(res["flow"][k][:len(flow)] - flow) / np.maximum(1.0, np.abs(flow))) <= 1e-11
