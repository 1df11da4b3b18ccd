"""Benchmark of the NRG hot path on B200.

One step = one full run of the reference's driver (main.F90) on the SIAM workload with
N_keep = 4096: Lambda=2, U=0.3, Gamma=0.03, eps_d=-0.15, 60 NRG iterations (sectors of
order up to ~1300), then the backward reduced density matrices and the T=0 CFS spectrum
on the reference's 1000-bins-per-decade grid, all in FP64.  Metric: NRG iterations per
second (60 per step), whole job.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

* value: device-resident run (nrg_run), inputs resident, timed with CUDA events on the
  stream the library launches on, barrier + synchronize on both sides, max over ranks.
* forward_only: the same sweep without the density matrices and the spectrum.
* bookkeeping: one forward sweep with the per-state bookkeeping between iterations
  (truncation, the next basis records and row lists, the kept energies) on the device,
  the default, and one with it on the host (NRG_HOST_TABLES=1): iterations/s, kernel
  launches and host<->device bytes per iteration.
* e2e: the same metric through the drop-in entry points with host arrays (every routine
  copies its module arrays host->device and back, as a Fortran caller would), with the
  caller's arrays page-locked; e2e.pageable: the same with pageable arrays (a Fortran
  allocatable), which the routines copy whole.
* roofline: the kernel with the largest share of device time, k_tri_cluster (Householder
  tridiagonalisation of the sectors of order > 128): algorithmic flops sum_s 4/3 d_s^3
  per launch over its event-timed launch duration, against a cuBLAS DGEMM peak measured
  here (the FP64 ceiling; tcgen05 has no FP64 kind); traffic = DRAM bytes per launch of an
  ncu capture of this workload, read from profiles/roofline_traffic.json (null without
  it).  "eigensolver" gives the same for the whole eigensolver of an iteration
  (sum_s (4/3+2) d_s^3 over the event-timed window).
* cpu_baseline: the oracle (numpy/scipy port of the reference path, OpenBLAS on all host
  threads) on two full-size iterations of the same chain with their backward density
  matrices and CFS spectrum (a bounded sample of the metric's scope).
* --impl reference: the oracle port on the same scope, rank 0 only: K steps, one
  full-size NRG iteration each (prepareBasis, dsyev per sector, truncation, both
  invariant-matrix routines) with its density-matrix and CFS steps, on a window of the
  headline chain
  whose last iteration is the window's last; W warm-up steps = W untimed full-size
  forward iterations.  The reference itself cannot be built here (Fortran, MPI, MKL).
* n_keep_2048: the N_keep = 2048 SIAM workload (Lambda=2, U=0.2, Gamma=0.02,
  eps_d=-0.1, 60 iterations), one warm-up and two event-timed sweeps.
* fdm: that workload with the full-density-matrix spectrum and density matrices at
  T = 1e-6 (the workload table's temperature; no reference counterpart: the reference's
  spectrum is the T = 0 CFS one), one warm-up and two event-timed sweeps.
* two_orbital_window: the two-orbital Hund model at N_keep = 8192 (16 local states),
  iterations -1..3 of its chain (sectors of order up to ~8,800), forward sweep only.
* many_instance: independent impurity models side by side (nrg_run_batch): the 27 draws
  with N_keep <= 1024 of the seeded 64-SIAM sweep (50 iterations each, T=0 CFS), run one
  at a time and then 8 in flight; wall clock around each batch with the device
  synchronised; with N ranks the instances are dealt to the ranks by the greedy cost
  rule and the slowest rank's time counts.
* many_instance_full: the many-instance workload itself: all 64 draws (N_keep from
  {512, 1024, 2048, 4096}) with the full-density-matrix spectrum at T = 1e-5, 8 in
  flight, each instance's storage released when it ends; wall clock around the batch.
Multi-GPU: one NRG instance does not shard (one GPU per instance), so N ranks run N
replicas of the headline workload; the many-instance sample is partitioned instead.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "nrg-mpi_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

WORKLOAD = dict(U=0.3, Gamma=0.03, eps_d=-0.15, Lambda=2.0, n_keep=4096, n_iterations=60)
WORKLOAD_NAME = ("SIAM flat band Lambda=2.0 U=0.3 Gamma=0.03 eps_d=-0.15 N_keep=4096, "
                 "60 NRG iterations + backward RDM + T=0 CFS spectrum (1000 bins/decade)")
SECOND = dict(U=0.2, Gamma=0.02, eps_d=-0.1, Lambda=2.0, n_keep=2048, n_iterations=60)
METRIC = "NRG iterations/s (full sweep + RDM + CFS spectrum, FP64, eig err <= 1e-12)"
# DRAM bytes per launch of the roofline kernel, from an ncu capture of this workload
TRAFFIC_FILE = os.path.join(ROOT, "profiles", "roofline_traffic.json")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-many", action="store_true")
    p.add_argument("--no-fdm", action="store_true")
    p.add_argument("--no-nk2048", action="store_true")
    p.add_argument("--no-pageable", action="store_true")
    p.add_argument("--no-two-orbital", action="store_true")
    p.add_argument("--no-many-full", action="store_true", help="skip the 64-instance FDM sweep")
    p.add_argument("--e2e-steps", type=int, default=3)
    # profiling helpers: a shorter sweep of the same model (not the headline workload)
    p.add_argument("--iterations", type=int, default=None)
    p.add_argument("--n-keep", type=int, default=None)
    a = p.parse_args()
    if a.iterations is not None:
        WORKLOAD["n_iterations"] = a.iterations
    if a.n_keep is not None:
        WORKLOAD["n_keep"] = a.n_keep
    return a


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")),
            int(os.environ.get("WORLD_SIZE", "1")))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.path = tempfile.mktemp(prefix="clocks_", suffix=".csv")
        self.proc = None

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), float(parts[3]), parts[5:9]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i, v in enumerate(r[3]) if v.lower() == "active"})
        loaded = [r[0] for r in rows if r[2] > 200.0] or [r[0] for r in rows]
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def fp64_peak_tflops(torch, device):
    """cuBLAS DGEMM throughput measured here (the FP64 roofline denominator)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=device)
    b = torch.randn(n, n, dtype=torch.float64, device=device)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize(device)
    best = float("inf")
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e) * 1e-3)
    del a, b
    return 2.0 * n ** 3 / best / 1e12


def many_instance(torch, dev, rank, world, dist, concurrency=8):
    """Independent instances side by side: the N_keep <= 1024 draws of the 64-SIAM sweep."""
    from nrg_b200 import Context, run_batch, sweep
    sample = [x for x in sweep.sweep_instances() if x.n_keep <= 1024]
    share = sweep.rank_share(sample, rank, world)
    ctxs = []
    try:
        for x in share:
            c = Context(dev.index)
            c.set_model(x.build())
            ctxs.append(c)
        run_batch(ctxs, spectrum=True, concurrency=concurrency)   # allocates every context's storage
        times = {}
        for conc in (1, concurrency):
            if dist is not None:
                dist.barrier()
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            res, _ = run_batch(ctxs, spectrum=True, concurrency=conc)
            torch.cuda.synchronize(dev)
            dt = time.perf_counter() - t0
            if dist is not None:
                t = torch.tensor([dt], device=dev, dtype=torch.float64)
                dist.all_reduce(t, op=dist.ReduceOp.MAX)
                dt = float(t.item())
            times[conc] = dt
    finally:
        for c in ctxs:
            c.close()
    its = sum(x.n_iterations for x in sample)
    return {"workload": f"{len(sample)} SIAMs of the seeded 64-instance draw (seed {sweep.SWEEP_SEED}) with "
                        "N_keep <= 1024, Lambda=2, 50 NRG iterations each + RDM + T=0 CFS spectrum",
            "instances": len(sample), "iterations": its, "unit": "iterations/s",
            "sequential": its / times[1], "batched": its / times[concurrency], "concurrency": concurrency,
            "ranks": world, "timing": "wall clock around each batch, device synchronised, max over ranks"}


def second_workload(torch, dev, local, stream, fdm_temperature=None):
    """The N_keep = 2048 workload: one warm-up and two sweeps, CUDA events on the library's
    stream (T = 0 CFS spectrum, or with fdm_temperature the FDM spectrum at that T); the
    context's storage is released afterwards."""
    from nrg_b200 import Context, model
    inp = model.siam(**SECOND)
    n_it = inp.numberOfIteration - inp.indexOfFirstIteration + 1
    T = fdm_temperature or 0.0
    c = Context(local)
    try:
        c.set_model(inp)
        c.set_stream(stream.cuda_stream)
        c.run(spectrum=True, temperature=T)
        torch.cuda.synchronize(dev)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ph = []
        s.record(stream)
        for _ in range(2):
            r = c.run(spectrum=True, temperature=T)
            ph.append(r["phaseSeconds"].copy())
        e.record(stream)
        torch.cuda.synchronize(dev)
        ms = s.elapsed_time(e) / 2
        nbin = r["numberOfBin"]
        sums = [float(r["binPos"][m * nbin:(m + 1) * nbin, 1].sum() + r["binNeg"][m * nbin:(m + 1) * nbin, 1].sum())
                for m in range(inp.numberOfMatrix)]
        p = np.mean(np.array(ph), axis=0)
        out = {"workload": "SIAM Lambda=2.0 U=0.2 Gamma=0.02 eps_d=-0.1 N_keep=2048, 60 iterations + backward "
                           + ("RDM + T=0 CFS spectrum" if not T else f"density matrices + FDM spectrum at T={T}"),
               "ms_per_sweep": ms, "iterations_per_s": n_it * 1e3 / ms,
               "phase_seconds": {"nrg_sweep": float(p[0]), "rdm": float(p[1]), "spectrum": float(p[2])},
               "sum_rule": sums,
               "timing": "CUDA events on the library's stream, 2 sweeps after 1 warm-up"}
        if T:
            out["temperature"] = T
            out["shell_trace_max_dev"] = float(np.nanmax(np.abs(r["rdmTrace"] - 1.0)))
        return out
    finally:
        c.close()


def many_instance_full(torch, dev, rank, world, dist, concurrency=8, temperature=1e-5):
    """The many-instance workload: all 64 draws of the seeded sweep (N_keep from {512,
    1024, 2048, 4096}, 50 iterations) with the full-density-matrix spectrum at
    T = `temperature`, largest first, `concurrency` in flight, each context's storage
    released when its instance ends.  Untimed first: one instance of each N_keep (module
    load, the GEMM tuner's first launches); then all 64 timed."""
    from nrg_b200 import Context, run_batch, sweep
    inst = sorted(sweep.sweep_instances(), key=lambda x: -x.cost())
    share = sweep.rank_share(inst, rank, world)
    ctxs = []
    try:
        for x in share:
            c = Context(dev.index)
            c.set_model(x.build())
            ctxs.append(c)
        warm, seen = [], set()
        for c, x in zip(ctxs, share):
            if x.n_keep not in seen:
                seen.add(x.n_keep)
                warm.append(c)
        run_batch(warm, spectrum=True, concurrency=concurrency, release=True, temperature=temperature)
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        res, _ = run_batch(ctxs, spectrum=True, concurrency=concurrency, release=True, temperature=temperature)
        torch.cuda.synchronize(dev)
        dt = time.perf_counter() - t0
        if dist is not None:
            t = torch.tensor([dt], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            dt = float(t.item())
    finally:
        for c in ctxs:
            c.close()
    sums = []
    for r in res:
        nbin = r["numberOfBin"]
        sums += [abs(float(r["binPos"][m * nbin:(m + 1) * nbin, 1].sum()
                           + r["binNeg"][m * nbin:(m + 1) * nbin, 1].sum()) - 1.0) for m in range(2)]
    its = sum(x.n_iterations for x in inst)
    return {"workload": f"all {len(inst)} SIAMs of the seeded draw (seed {sweep.SWEEP_SEED}), N_keep from "
                        "{512, 1024, 2048, 4096}, Lambda=2, 50 NRG iterations each + density matrices + FDM "
                        f"spectrum at T={temperature}",
            "instances": len(inst), "iterations": its, "seconds": dt, "iterations_per_s": its / dt,
            "concurrency": concurrency, "ranks": world, "sum_rule_max_dev": max(sums) if sums else None,
            "timing": "wall clock around the batch, device synchronised, max over ranks; storage released per "
                      "instance; one instance of each N_keep run untimed first"}


def two_orbital_window(torch, dev, local, stream):
    """The two-orbital Hund model at N_keep = 8192 (16 local states, sectors of order up to
    ~8,800), its first 5 iterations (-1..3), forward sweep only: one warm-up and one
    event-timed sweep; the context's storage is released afterwards."""
    from nrg_b200 import Context, model
    inp = model.config(4, n_iterations=5)
    inp.flag_spectrum = False
    n_it = inp.numberOfIteration - inp.indexOfFirstIteration + 1
    c = Context(local)
    try:
        c.set_model(inp)
        c.set_stream(stream.cuda_stream)
        c.run(spectrum=False)
        torch.cuda.synchronize(dev)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        r = c.run(spectrum=False)
        e.record(stream)
        torch.cuda.synchronize(dev)
        ms = s.elapsed_time(e)
        return {"workload": "two-orbital Hund model U=0.2 J=0.02 Gamma=0.015 Lambda=3 N_keep=8192, iterations "
                            "-1..3 (a window of the 40-iteration chain), forward sweep only",
                "ms_per_window": ms, "iterations_per_s": n_it * 1e3 / ms,
                "kept": [int(k) for k in r["kept"]],
                "states_before_truncation": [int(k) for k in r["numberOfBasisFull"]],
                "timing": "CUDA events on the library's stream, 1 window after 1 warm-up"}
    finally:
        c.close()


def oracle_window(n_full, warmup=0):
    """The oracle port over the scope of the headline's metric: forward NRG iterations, the
    backward reduced density matrices and the CFS spectrum, on a window of the same chain
    (the headline chain cut so that its last n_full iterations are the full-size ones:
    every iteration from the first truncated one to the last, whose sizes and per-iteration
    work are those of the 60-iteration sweep).  The iterations before full size (five,
    cheap) run untimed; `warmup` full-size forward iterations of another window run first,
    untimed.  Returns (iterations/s, seconds, first and last timed iteration, states per
    iteration)."""
    from nrg_b200 import model
    from oracle import nrg_oracle as O

    def window(n):
        # the first full-size iteration: before it no truncation happens, so the basis grows
        # by nOps per iteration from the initial one
        probe = model.siam(**WORKLOAD)
        k, nb = 0, probe.numberOfBasis
        while nb < WORKLOAD["n_keep"]:
            nb *= probe.numberOfOperation
            k += 1
        last = probe.indexOfFirstIteration + k + n - 1
        inp = model.siam(**dict(WORKLOAD, n_iterations=last + 2))   # numberOfIteration = n_iterations - 2
        d = tempfile.mkdtemp(prefix="nrg_cpu_")
        model.write_inputs(inp, d)
        st = O.State(d)
        it = st.first
        while st.numberOfBasis_old < st.truncation and it <= st.nIter:
            O.nrg_iteration(st, it)    # grow to full size (untimed)
            it += 1
        return st, it

    if warmup > 0:
        st, it = window(warmup)
        for N in range(it, st.nIter + 1):
            O.nrg_iteration(st, N)
    st, it0 = window(n_full)
    t0 = time.perf_counter()
    for N in range(it0, st.nIter + 1):                # main.F90:175-177
        O.nrg_iteration(st, N)
    if st.flag_truncation:                            # main.F90:188-201
        O.initialize_reduced_density(st)
        O.reduced_density_matrix_calculation(st)
    for N in range(st.startTrancation, st.nIter + 1):   # main.F90:204-224
        O.cfs_spectrum_calculation(st, N)
    dt = time.perf_counter() - t0
    n = st.nIter - it0 + 1
    return n / dt, dt, it0, st.nIter, int(st.numberOfBasis_full)


def roofline_traffic():
    """DRAM bytes per launch of the roofline kernel on this workload (ncu), if captured."""
    try:
        with open(TRAFFIC_FILE) as f:
            t = json.load(f)
        return float(t["bytes_per_launch"]), os.path.relpath(TRAFFIC_FILE, ROOT)
    except (OSError, ValueError, KeyError):
        return None, None


def headline_config(world):
    """The `config` object of both arms' JSON lines."""
    return {"workload": WORKLOAD_NAME, "n_keep": WORKLOAD["n_keep"],
            "iterations": WORKLOAD["n_iterations"], "parallelism": f"replicas x{world}",
            "l2": "working set > L2: each step writes ~20 GB of eigenvector blocks and spectral matrices"}


def reference_arm(args):
    rank, _, world = dist_env()
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("gloo")
        if rank != 0:
            dist.barrier()
            dist.destroy_process_group()
            return
    # K timed steps = K full-size NRG iterations with their backward density matrices and
    # CFS spectrum (~10 s each on 16 host threads); W warm-up steps = W untimed full-size
    # forward iterations (K = 20, W = 5: about four and a half minutes in all)
    warm = max(0, args.warmup)
    v, dt, i0, i1, nbf = oracle_window(max(1, args.steps), warmup=warm)
    n = i1 - i0 + 1
    cores = os.cpu_count()
    sample = (f"full-size NRG iterations {i0}..{i1} of the headline chain (nb ~ {nbf} each) with their "
              f"backward density matrices and CFS spectrum, the window's last iteration as the last; "
              f"{dt:.1f} s, numpy/scipy-OpenBLAS oracle on {cores} host threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "iterations/s",
        "n_gpus": args.gpus, "steps": n, "warmup": warm,
        "ms_per_step": dt / n * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (generated Wilson chain and impurity tables)",
        "config": headline_config(world),
        "scope": ("one step = one full-size NRG iteration (prepareBasis, dsyev per sector, truncation, both "
                  "invariant-matrix routines) plus its step of the backward density matrices and of the CFS "
                  "spectrum; the b200 arm's value also counts the five cheap iterations before full size"),
        "cpu_baseline": {"value": v, "unit": "iterations/s", "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": "iterations/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    import torch
    rank, local, world = dist_env()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=dev)
    from nrg_b200 import Context, model
    inp = model.siam(**WORKLOAD)
    n_it = inp.numberOfIteration - inp.indexOfFirstIteration + 1
    peak = fp64_peak_tflops(torch, dev) if rank == 0 else None
    torch.cuda.empty_cache()
    free0 = torch.cuda.mem_get_info(dev)[0]
    ctx = Context(local)
    ctx.set_model(inp)
    stream = torch.cuda.current_stream(dev)
    ctx.set_stream(stream.cuda_stream)
    for _ in range(args.warmup):
        res = ctx.run(spectrum=True)
    torch.cuda.synchronize(dev)
    # device memory the library holds for one instance of the workload (stores and workspaces)
    device_gb = (free0 - torch.cuda.mem_get_info(dev)[0]) / 1e9
    ctx.set_profiling(True)
    ctx.reset_stats()
    l0 = ctx.launch_count
    phases = []
    with ClockSampler(local) as clk:
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        for _ in range(args.steps):
            res = ctx.run(spectrum=True)
            phases.append(res["phaseSeconds"].copy())
        e.record(stream)
        torch.cuda.synchronize(dev)
        if dist is not None:
            dist.barrier()
    elapsed = s.elapsed_time(e) * 1e-3
    launches = ctx.launch_count - l0
    stats = ctx.stats()
    ctx.set_profiling(False)
    t_max = elapsed
    if dist is not None:
        t = torch.tensor([elapsed], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_max = float(t.item())
    value = n_it * args.steps * world / t_max
    # the forward sweep alone (the reference arm's scope), one event-timed sweep
    sf, ef = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sf.record(stream)
    ctx.run(spectrum=False)
    ef.record(stream)
    torch.cuda.synchronize(dev)
    forward_only = {"value": n_it * 1e3 / sf.elapsed_time(ef), "unit": "iterations/s",
                    "timing": "one sweep without density matrices and spectrum, CUDA events"}

    def forward_sweep(host_tables):
        # one event-timed forward sweep with the per-state bookkeeping on the device (the
        # default) or on the host (NRG_HOST_TABLES=1), no energy-flow output
        if host_tables:
            os.environ["NRG_HOST_TABLES"] = "1"
        try:
            ctx.run(spectrum=False, flow_stride=0)
            torch.cuda.synchronize(dev)
            ctx.reset_stats()
            l0 = ctx.launch_count
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            ctx.run(spectrum=False, flow_stride=0)
            b.record(stream)
            torch.cuda.synchronize(dev)
            st = ctx.stats()
            return {"iterations_per_s": n_it * 1e3 / a.elapsed_time(b),
                    "launches_per_iteration": (ctx.launch_count - l0) / n_it,
                    "h2d_bytes_per_iteration": int(st["h2d_bytes"]) // n_it,
                    "d2h_bytes_per_iteration": int(st["d2h_bytes"]) // n_it}
        finally:
            os.environ.pop("NRG_HOST_TABLES", None)

    bookkeeping = {"what": "forward sweep of the headline workload with the per-state bookkeeping "
                           "(truncation, basis records, row lists, kept energies) on the device and on "
                           "the host; CUDA events, one sweep each",
                   "device": forward_sweep(False), "host": forward_sweep(True)}

    def drop_in(pageable, steps):
        # one untimed run allocates the emulated caller's module arrays, then K timed runs
        r = ctx.run(spectrum=True, host_drop_in=True, host_pageable=pageable)
        torch.cuda.synchronize(dev)
        ctx.reset_stats()
        if dist is not None:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(steps):
            r = ctx.run(spectrum=True, host_drop_in=True, host_pageable=pageable)
        torch.cuda.synchronize(dev)
        dt = (time.perf_counter() - t0) / steps
        st2 = ctx.stats()
        if dist is not None:
            t = torch.tensor([dt], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            dt = float(t.item())
        same = float(max(np.max(np.abs(r["binPos"][:, 1] - res["binPos"][:, 1])),
                         np.max(np.abs(r["binNeg"][:, 1] - res["binNeg"][:, 1]))))
        return {"value": n_it * world / dt, "unit": "iterations/s",
                "h2d_bytes_per_step": int(st2["h2d_bytes"]) // steps,
                "d2h_bytes_per_step": int(st2["d2h_bytes"]) // steps, "steps": steps,
                "max_bin_diff_vs_device_resident": same}

    # end to end through the drop-in entry points with host arrays
    e2e = None
    if not args.no_e2e:
        k = max(1, min(args.steps, args.e2e_steps))
        e2e = drop_in(False, k)
        e2e["path"] = ("drop-in entry points with host arrays (the Fortran caller's data flow), module "
                       "arrays in page-locked host memory allocated in one untimed run; host<->device "
                       "copies inside the timed region")
        e2e["timing"] = "wall clock around the runs, device synchronised, max over ranks"
        # where the drop-in time goes: one more run with the parts timed apart (the stream
        # is drained between them, so they do not overlap; not part of the timed runs)
        ctx.reset_stats()
        ctx.set_profiling(True)
        ctx.run(spectrum=True, host_drop_in=True)
        ctx.set_profiling(False)
        sb = ctx.stats()
        e2e["breakdown_seconds"] = {
            "entry_staging_in": sb["entry_in_s"], "entry_device": sb["entry_compute_s"],
            "entry_copy_out": sb["entry_out_s"], "replay_host": sb["replay_host_s"],
            "entry_calls": int(sb["entry_calls"]),
            "timing": "one untimed sweep with profiling on, host wall clock, stream drained between parts"}
        if not args.no_pageable:
            pg = drop_in(True, 1)
            pg["path"] = "the same with the module arrays in pageable memory (a Fortran allocatable)"
            e2e["pageable"] = pg
    ctx.release_storage()   # the headline's device storage; the model stays set
    nk2048 = None if args.no_nk2048 else second_workload(torch, dev, local, stream)
    fdm = None if args.no_fdm else second_workload(torch, dev, local, stream, fdm_temperature=1e-6)
    many = None if args.no_many else many_instance(torch, dev, rank, world, dist)
    two = None if args.no_two_orbital else two_orbital_window(torch, dev, local, stream)
    many_full = None if args.no_many_full else many_instance_full(torch, dev, rank, world, dist)
    if rank == 0:
        clocks = clk.summary()
        nbin = res["numberOfBin"]
        sums = [float(res["binPos"][m * nbin:(m + 1) * nbin, 1].sum() + res["binNeg"][m * nbin:(m + 1) * nbin, 1].sum())
                for m in range(inp.numberOfMatrix)]
        ph = np.mean(np.array(phases), axis=0)
        syev_avg_s = stats["syev_ms"] * 1e-3 / max(stats["syev_launches"], 1)
        flops_per_launch = stats["syev_flops"] / max(stats["syev_launches"], 1)
        achieved = flops_per_launch / syev_avg_s / 1e12 if syev_avg_s > 0 else None
        tri_avg_s = stats["tri_ms"] * 1e-3 / max(stats["tri_launches"], 1)
        tri_flops = stats["tri_flops"] / max(stats["tri_launches"], 1)
        tri_ach = tri_flops / tri_avg_s / 1e12 if tri_avg_s > 0 else None
        traffic, traffic_src = roofline_traffic()
        cpu = None
        if not args.no_cpu:
            v, dt, i0, i1, nbf = oracle_window(2)
            cpu = {"value": v, "unit": "iterations/s", "cores": os.cpu_count(), "kind": "port",
                   "sample": f"full-size NRG iterations {i0}..{i1} of the same chain (nb ~ {nbf} each) with "
                             f"their backward density matrices and CFS spectrum (the window's last "
                             f"iteration as the last), {dt:.1f} s, numpy/scipy-OpenBLAS oracle on all host "
                             "threads"}
        line = {
            "metric": METRIC, "value": value, "unit": "iterations/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (generated Wilson chain and impurity tables)",
            "config": headline_config(world),
            "phase_seconds": {"nrg_sweep": float(ph[0]), "rdm": float(ph[1]), "cfs_spectrum": float(ph[2])},
            "spectrum_seconds": float(ph[2]),
            "forward_only": forward_only,
            "bookkeeping": bookkeeping,
            "device_memory_gb": device_gb,
            "sum_rule": sums,
            "gpu_launches": int(launches),
            "roofline": {"kernel": "k_tri_cluster (FP64 Householder tridiagonalisation of the sectors of "
                                   "order > 128, one thread-block cluster per sector)",
                         "bound": "tensor", "pipe": "fp64",
                         "achieved": tri_ach, "peak": peak, "unit": "TFLOP/s",
                         "frac": (tri_ach / peak) if (tri_ach and peak) else None,
                         "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (MEASURED_PEAKS.json has no "
                                        "FP64 figure)",
                         "flops_per_launch": tri_flops, "avg_launch_ms": tri_avg_s * 1e3,
                         "launches": int(stats["tri_launches"]),
                         "traffic": traffic, "traffic_source": traffic_src},
            "eigensolver": {"what": "all sectors of one iteration: tridiagonalisation, divide and conquer, "
                                    "back-transformation (three streams)",
                            "achieved": achieved, "unit": "TFLOP/s", "peak": peak,
                            "frac": (achieved / peak) if (achieved and peak) else None,
                            "flops_per_launch": flops_per_launch, "avg_window_ms": syev_avg_s * 1e3,
                            "windows": int(stats["syev_launches"])},
            "clocks": clocks,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "n_keep_2048": nk2048,
            "fdm": fdm,
            "many_instance": many,
            "two_orbital_window": two,
        }
        line["many_instance_full"] = many_full
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
