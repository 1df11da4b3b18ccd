"""The tridiagonalisation paths other than the default one (the full-column cluster kernel
on 8-block clusters), each through the large-sector parity test re-run in a child process
with the environment variable that selects it (read once per process):
* the multi-kernel path (two launches per column, then grouped-GEMM panel updates), which
  sectors too large for the cluster kernels' shared memory take: NRG_TRI_CLUSTER=0;
* the lower-triangle cluster kernel on 8-block clusters: NRG_TRI_SYM=1;
* the lower-triangle kernel on 16-block clusters: NRG_TRI_SYM=1 NRG_TRI_CLUSTER=16."""
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


@pytest.mark.parametrize("env,case", [
    ({"NRG_TRI_SYM": "1"}, "nkeep4096"),                            # lower triangle, 8 blocks
    ({"NRG_TRI_SYM": "1", "NRG_TRI_CLUSTER": "16"}, "nkeep4096"),   # lower triangle, 16 blocks
])
def test_large_sectors_through_the_other_cluster_kernels(env, case):
    # the N_keep = 4096 case reaches orders 1225 and 1308
    cmd = [sys.executable, "-m", "pytest", "-q", "-x", "-p", "no:cacheprovider",
           os.path.join(HERE, "test_gpu_parity.py") + f"::test_large_sector_diagonalization[{case}]"]
    r = subprocess.run(cmd, env=dict(os.environ, **env), cwd=os.path.dirname(HERE), capture_output=True,
                       text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    assert "1 passed" in r.stdout
