import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "nrg-mpi_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def ctx_factory():
    """Creates CUDA contexts through the C ABI (GPU tests only)."""
    from nrg_b200 import Context
    made = []

    def make(inp):
        c = Context(0)
        c.set_model(inp)
        made.append(c)
        return c

    yield make
    for c in made:
        c.close()
