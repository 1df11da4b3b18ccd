"""CPU tests of the C ABI library and the host-side logic (no compute without a GPU)."""
import ctypes
import os
import re

import numpy as np
import pytest

from nrg_b200 import model, load_library, LIB_PATH
from nrg_b200.abi import EXPORTS

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "nrg_b200.h")


def declared():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"NRG_API\s+[\w\s\*]+?\b(nrg_\w+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    lib = load_library()
    names = declared()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), f"{n} declared in nrg_b200.h but not exported"
    assert sorted(EXPORTS) == names, "abi.EXPORTS out of date"


def test_no_device_means_loud_failure():
    lib = load_library()
    h = ctypes.c_void_p()
    rc = lib.nrg_context_create(ctypes.byref(h), 0)
    if rc == 0:
        lib.nrg_context_destroy(h)
        pytest.skip("a CUDA device is present")
    assert rc == 5   # NRG_ERR_DEVICE: no CPU fallback
    assert b"CUDA device" in lib.nrg_last_error()
    # compute entry points refuse a missing context instead of computing on the host
    assert lib.nrg_run(None, None, None) == 1
    assert lib.nrg_diagonalization(None, 0, None) != 0


def test_status_strings():
    lib = load_library()
    assert lib.nrg_status_string(0) == b"ok"
    assert lib.nrg_status_string(6) == b"unsupported input"


def test_input_files_round_trip(tmp_path):
    inp = model.config(1, n_keep=64, n_iterations=8)
    model.write_inputs(inp, str(tmp_path))
    back = model.read_inputs(str(tmp_path))
    assert back.numberOfBasis == inp.numberOfBasis == 4
    assert back.numberOfOperation == 4 and back.numberOfConductionMatrix == 2
    assert np.array_equal(back.basis_output, inp.basis_output)
    assert np.array_equal(back.operation, inp.operation)
    assert np.array_equal(back.coefficient_diagonalization_type, inp.coefficient_diagonalization_type)
    assert np.allclose(back.invariant_matrix, inp.invariant_matrix, rtol=0, atol=0)
    assert np.allclose(back.chain_nondiagonal_raw, inp.chain_nondiagonal_raw, rtol=0, atol=0)
    assert np.array_equal(back.conservationBlock, inp.conservationBlock)


def test_wilson_chain_rescale():
    # read_initial_basis.F90:127-139 with z = 1: t_n / scale(n) -> 1 for large n, and the
    # hybridisation chain_nondiagonal(-1) is used as written
    inp = model.config(2, n_iterations=40)
    cd, cn, _ = inp.rescaled_chains()
    first = inp.indexOfFirstIteration
    assert cn[0, 0] == inp.chain_nondiagonal_raw[0, 0]
    assert abs(cn[30 - first, 0] - 1.0) < 1e-6
    for n in range(0, 10):
        assert abs(cn[n - first, 0] - inp.chain_nondiagonal_raw[n - first, 0] / inp.scale(n)) < 1e-14


def test_local_site_tables_are_fermionic():
    # the diagonalisation table couples |0>->|up> with +1 and |dn>->|updn> with -1 (SIAM)
    inp = model.siam(U=0.1, Gamma=0.01, n_keep=64, n_iterations=6)
    rows = {tuple(r[:3]): c for r, c in zip(inp.coefficient_diagonalization_type,
                                           inp.coefficient_diagonalization)}
    assert rows[(1, 2, 1)] == 1.0
    assert rows[(3, 4, 1)] == -1.0
    assert rows[(2, 4, 2)] == 1.0
    assert np.array_equal(inp.coefficient_invariant_matrix_spectrum[0], [1, -1, -1, 1])


def test_two_orbital_model_tables():
    inp = model.two_orbital_hund(n_keep=64, n_iterations=6)
    assert inp.numberOfOperation == 16 and inp.numberOfChain == 2
    assert inp.numberOfConductionMatrix == 4
    # every local creation operator appears once per (lower, upper) pair
    assert inp.numberOfCoefficient == 4 * 8
