"""The C++ restart.dat reader and writer (nrg-mpi_b200/csrc/restart.cu) on the CPU,
without a device: tests/restart_harness.cu, built here with nvcc and linked to restart.cu
alone, writes and reads back a synthetic stock; sets every 4-byte word of the file in
turn to 2^31-1 (counts and bounds are refused as a broken file, never an allocation
failure or an exception across the C ABI); cuts the file at every 7th byte (always
refused); and loads a file the oracle's saveRestart restatement wrote (the two
implementations of the layout agree)."""
import os
import shutil
import subprocess

import pytest

from oracle import nrg_oracle as O

from helpers import small_siam, write_case

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


@pytest.mark.skipif(not os.path.exists(NVCC) and shutil.which("nvcc") is None, reason="nvcc not available")
def test_restart_reader_and_writer_without_a_device(tmp_path):
    exe = str(tmp_path / "restart_harness")
    subprocess.run([NVCC if os.path.exists(NVCC) else "nvcc", "-std=c++17", "-O1", "-Wno-deprecated-gpu-targets",
                    "-o", exe, os.path.join(HERE, "restart_harness.cu"),
                    os.path.join(ROOT, "nrg-mpi_b200", "csrc", "restart.cu"), "-I", os.path.join(ROOT, "include")],
                   check=True, capture_output=True, timeout=600)
    d = write_case(small_siam(n_keep=48, n_iterations=14), str(tmp_path))
    full = O.run(d)
    path = str(tmp_path / "oracle_restart.dat")
    O.run_with_restart(d, save_path=path, stop_before=full.startTrancation + 2)
    args = [path, full.nIter, full.first, full.nVar, full.nMat, full.nCM, full.nChain, full.nOps, full.numberOfBin]
    r = subprocess.run([exe] + [str(a) for a in args], capture_output=True, text=True, timeout=300, cwd=str(tmp_path))
    assert r.returncode == 0, r.stdout + r.stderr
    assert "round trip: ok" in r.stdout and "exceptions 0" in r.stdout
    assert "truncations refused" in r.stdout and "accepted 0" in r.stdout.split("truncations")[1]
    assert "oracle-written file: ok" in r.stdout
