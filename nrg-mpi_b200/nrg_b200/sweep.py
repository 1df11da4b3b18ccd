"""Many-instance parameter sweeps: independent impurity models spread over GPUs and run side
by side on each GPU.

The reference runs one impurity per MPI job and balances the symmetry sectors of one
iteration over its ranks with a greedy cost rule (loadbalanceDiagonalization2,
loadbalance.F90:102-186: sectors by decreasing d^3, each to the least loaded rank).
Here the unit of work is a whole instance: instances never exchange data, so the
instances are dealt to the ranks by the same greedy rule on an instance cost, with no
collective on the data path, and each rank runs its share through nrg_run_batch
(concurrent instances, one CUDA stream each).

The sweep of the many-instance workload: 64 single-impurity Anderson models on a flat
band with Lambda = 2, 50 NRG iterations, U uniform in [0.05, 0.5], Gamma log-uniform in
[0.005, 0.05], eps_d = -U/2 + delta with delta uniform in [-0.02, 0.02], N_keep drawn
from {512, 1024, 2048, 4096}, all from numpy's default_rng(seed).
"""
from __future__ import annotations

import dataclasses
from typing import Dict, List, Sequence

import numpy as np

from . import model

SWEEP_SEED = 20261203
NKEEP_CHOICES = (512, 1024, 2048, 4096)


@dataclasses.dataclass(frozen=True)
class Instance:
    """One impurity model of a sweep (the arguments of model.siam)."""
    index: int
    U: float
    Gamma: float
    eps_d: float
    n_keep: int
    Lambda: float = 2.0
    n_iterations: int = 50

    def cost(self) -> float:
        """Work estimate: the eigensolves dominate and their flops grow like the cube of
        the kept-state count, once per iteration (the d^3 load of loadbalance.F90:124
        applied to the largest block size, which scales with N_keep)."""
        return float(self.n_iterations) * float(self.n_keep) ** 3

    def device_bytes(self) -> float:
        """Device storage of one run: kept for every iteration, the dense d-dagger matrices
        of the kept states ((1.2 N_keep)^2 x 2 doubles, the reference's layout) and the
        eigenvector blocks (about a fifth of that), plus ~1 GB of workspace."""
        k = 1.2 * self.n_keep
        return self.n_iterations * 1.2 * k * k * 2 * 8 + 1e9

    def build(self):
        return model.siam(U=self.U, Gamma=self.Gamma, eps_d=self.eps_d, Lambda=self.Lambda,
                          n_keep=self.n_keep, n_iterations=self.n_iterations)


def sweep_instances(count: int = 64, seed: int = SWEEP_SEED, n_iterations: int = 50,
                    nkeep_choices: Sequence[int] = NKEEP_CHOICES, Lambda: float = 2.0) -> List[Instance]:
    """The seeded parameter draw of the many-instance workload."""
    rng = np.random.default_rng(seed)
    U = rng.uniform(0.05, 0.5, count)
    G = 10.0 ** rng.uniform(np.log10(0.005), np.log10(0.05), count)
    delta = rng.uniform(-0.02, 0.02, count)
    nk = rng.choice(np.asarray(nkeep_choices, dtype=np.int64), count)
    return [Instance(i, float(U[i]), float(G[i]), float(-U[i] / 2 + delta[i]), int(nk[i]), Lambda, n_iterations)
            for i in range(count)]


def partition(costs: Sequence[float], nparts: int) -> List[List[int]]:
    """Greedy longest-processing-time assignment (loadbalance.F90:102-186): items by
    decreasing cost (ties by index), each to the part with the smallest load (ties by
    part number).  Every part lists its items by decreasing cost."""
    if nparts < 1:
        raise ValueError("nparts must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * nparts
    parts: List[List[int]] = [[] for _ in range(nparts)]
    for i in order:
        p = min(range(nparts), key=lambda q: (load[q], q))
        parts[p].append(i)
        load[p] += float(costs[i])
    return parts


def rank_share(instances: Sequence[Instance], rank: int, world: int) -> List[Instance]:
    """The instances this rank runs (largest cost first)."""
    parts = partition([x.cost() for x in instances], world)
    return [instances[i] for i in parts[rank]]


def memory_concurrency(share: Sequence[Instance], free_bytes: float, limit: int = 8,
                       fraction: float = 0.85) -> int:
    """Instances in flight such that the largest ones fit in ``fraction`` of the free
    device memory together (instances start largest first)."""
    sizes = sorted((x.device_bytes() for x in share), reverse=True)
    c, used = 0, 0.0
    for b in sizes[:max(1, limit)]:
        if c > 0 and used + b > fraction * free_bytes:
            break
        used += b
        c += 1
    return max(1, c)


def run_share(share: Sequence[Instance], device: int = 0, concurrency: int = 8,
              spectrum: bool = True, contexts=None) -> Dict[int, dict]:
    """Runs one rank's instances on one GPU through nrg_run_batch (largest first, each
    instance's device storage released when it ends, no more in flight than the free
    memory holds); returns the result of every instance by its sweep index.
    ``contexts`` (optional) reuses contexts whose models are already set, one per
    instance in ``share`` order."""
    from .abi import Context, run_batch
    order = sorted(range(len(share)), key=lambda i: (-share[i].cost(), share[i].index))
    own = contexts is None
    ctxs = list(contexts) if contexts is not None else []
    try:
        if own:
            for x in share:
                c = Context(device)
                c.set_model(x.build())
                ctxs.append(c)
        try:
            import torch
            with torch.cuda.device(device):
                free_b = float(torch.cuda.mem_get_info()[0])
        except Exception:
            free_b = 64e9
        conc = memory_concurrency([share[i] for i in order], free_b, concurrency)
        results, _ = run_batch([ctxs[i] for i in order], spectrum=spectrum, concurrency=conc, release=True)
        return {share[i].index: r for i, r in zip(order, results)}
    finally:
        if own:
            for c in ctxs:
                c.close()
