"""The multi-kernel tridiagonalisation (two launches per column, then grouped-GEMM panel
updates), which sectors too large for the one-launch cluster kernel's shared memory
take (order above ~1500): the large-sector parity test re-run in a child process with
NRG_TRI_CLUSTER=0, which sends every sector of order > 128 down that path (the variable
is read once per process)."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def test_large_sectors_through_the_multi_kernel_tridiagonalisation():
    env = dict(os.environ, NRG_TRI_CLUSTER="0")
    cmd = [sys.executable, "-m", "pytest", "-q", "-x", "-p", "no:cacheprovider",
           os.path.join(HERE, "test_gpu_parity.py") + "::test_large_sector_diagonalization[nkeep512]"]
    r = subprocess.run(cmd, env=env, cwd=os.path.dirname(HERE), capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    assert "1 passed" in r.stdout
