"""Writes the golden fixtures of the benchmarked workloads from the CPU oracle.

The reference ships no outputs, so the oracle (a restatement of the reference's routines,
``oracle/nrg_oracle.py``) produces them once on the CPU; the GPU tests then compare the
library's whole runs with these files instead of re-running the oracle at full size.

Workloads (``nrg_b200.model.config``):

* ``siam_nkeep2048.npz``  SIAM Lambda=2.0 U=0.2 Gamma=0.02 eps_d=-0.1, N_keep=2048, all 60
  iterations (-1..58), backward reduced density matrices and the T = 0 CFS spectrum;
* ``siam_nkeep4096.npz`` SIAM Lambda=2.0 U=0.3 Gamma=0.03 eps_d=-0.15, N_keep=4096 (the
  bench headline's workload), all 60 iterations (-1..58), backward reduced density
  matrices and the T = 0 CFS spectrum (about 15 minutes and 30 GB of host memory for the
  oracle);
* ``two_orbital_nkeep8192_n5.npz`` the two-orbital Hund model (U=0.2, J=0.02, Gamma=0.015
  per orbital, Lambda=3, 16 local states, N_keep=8192), its first 5 iterations (-1..3),
  forward sweep only (no spectrum): sectors of order up to ~8,800, tied sort keys.

Stored per iteration: the kept count, the number of states before truncation, the
ground-state energy (eigenvalue(1) before the shift), the lowest ``FLOW`` kept energies
(energy flow), calcThermo's (Cn, Sn, Xn); per backward step the density-matrix trace; the
nonzero bins of both spectral arrays (indices and weights); the bin count and the
truncation start.  Usage: ``python tests/golden/make_golden.py [name ...]``.
"""
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for _p in (ROOT, os.path.join(ROOT, "nrg-mpi_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

from nrg_b200 import model  # noqa: E402
from oracle import nrg_oracle as O  # noqa: E402

FLOW = 64

def _two_orbital_window():
    inp = model.config(4, n_iterations=5)
    inp.flag_spectrum = False       # forward sweep only
    return inp


CASES = {
    "siam_nkeep2048": lambda: model.config(2),
    "siam_nkeep4096": lambda: model.config(3),
    "two_orbital_nkeep8192_n5": _two_orbital_window,
}


def golden(inp) -> dict:
    d = tempfile.mkdtemp(prefix="nrg_golden_")
    model.write_inputs(inp, d)
    st = O.State(d)
    nfull = {}
    for it in range(st.first, st.nIter + 1):        # main.F90:175-177, as nrg_oracle.run
        O.nrg_iteration(st, it)
        nfull[it] = st.numberOfBasis_full
    if st.flag_spectrum:
        if st.flag_truncation:                        # main.F90:188-201
            O.initialize_reduced_density(st)
            O.reduced_density_matrix_calculation(st)
        for it in range(st.startTrancation, st.nIter + 1):
            O.cfs_spectrum_calculation(st, it)
    its = list(range(st.first, st.nIter + 1))
    flow = np.full((len(its), FLOW), np.nan)
    for k, i in enumerate(its):
        f = st.flow[i][:FLOW]
        flow[k, :len(f)] = f
    tr = np.full(st.nIter + 1, np.nan)
    for N, v in st.rdm_trace.items():
        tr[N] = v
    out = dict(
        first=st.first, nIter=st.nIter, startTrancation=st.startTrancation, numberOfBin=st.numberOfBin,
        nMat=st.nMat,
        kept=np.array([st.kept[i] for i in its], dtype=np.int32),
        numberOfBasisFull=np.array([nfull[i] for i in its], dtype=np.int32),
        groundStateEnergy=np.array([st.ground_state_energy[i] for i in its]),
        flow=flow,
        thermo=np.array([st.thermo[i] for i in its]),
        rdmTrace=tr,
    )
    for name, arr in (("binPos", st.binPos), ("binNeg", st.binNeg)):
        w = arr[:, 1]
        nz = np.nonzero(w)[0].astype(np.int32)
        out[name + "_index"] = nz
        out[name + "_weight"] = w[nz]
    return out


def main(names):
    for name in names:
        t0 = time.time()
        g = golden(CASES[name]())
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **g)
        print(f"{name}: {time.time() - t0:.0f} s, {os.path.getsize(path)} bytes", flush=True)


if __name__ == "__main__":
    main(sys.argv[1:] or list(CASES))
