"""B200-native NRG hot path (sector diagonalisation, invariant matrices, backward reduced
density matrices and CFS spectrum) behind the C ABI of include/nrg_b200.h."""
from . import model
from .abi import Context, NrgError, load_library, prepare_basis, run_batch, truncate, LIB_PATH, EXPORTS

__all__ = ["model", "Context", "NrgError", "load_library", "prepare_basis", "run_batch", "truncate", "LIB_PATH", "EXPORTS"]
