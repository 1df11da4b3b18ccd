"""Host logic of the many-instance sweep: the seeded draw, the greedy partition of
instances over ranks (loadbalance.F90:102-186 applied to whole instances) and the
two-rank split over a gloo process group (CPU only)."""
import os
import socket

import numpy as np
import pytest

from nrg_b200 import sweep


def _reference_lpt(costs, nproc):
    """loadbalanceDiagonalization2 (loadbalance.F90:120-150) line by line: the heaviest
    remaining job (first index on ties) to the least busy process (first on ties)."""
    load = [float(c) for c in costs]
    busy = [0.0] * nproc
    owner = [-1] * len(costs)
    for _ in range(len(costs)):
        jmax, loadmax = 0, None
        for j in range(len(costs)):
            if j == 0 or loadmax < load[j]:
                loadmax, jmax = load[j], j
        pmin, busymin = 0, None
        for p in range(nproc):
            if p == 0 or busymin > busy[p]:
                busymin, pmin = busy[p], p
        busy[pmin] += load[jmax]
        load[jmax] = 0.0
        owner[jmax] = pmin
    return owner


@pytest.mark.parametrize("nparts", [1, 2, 3, 8])
def test_partition_matches_reference_greedy_rule(nparts):
    rng = np.random.default_rng(5)
    costs = rng.choice([1.0, 8.0, 27.0, 64.0], 40) * rng.integers(1, 4, 40)
    parts = sweep.partition(costs, nparts)
    owner = _reference_lpt(costs, nparts)
    for p, items in enumerate(parts):
        for i in items:
            assert owner[i] == p
    flat = sorted(i for items in parts for i in items)
    assert flat == list(range(len(costs)))
    for items in parts:
        c = [costs[i] for i in items]
        assert c == sorted(c, reverse=True)
    loads = [sum(costs[i] for i in items) for items in parts]
    assert max(loads) <= sum(costs) / nparts + max(costs) + 1e-9


def test_sweep_draw_is_seeded_and_in_range():
    a = sweep.sweep_instances()
    b = sweep.sweep_instances()
    assert a == b and len(a) == 64
    for x in a:
        assert 0.05 <= x.U <= 0.5
        assert 0.005 <= x.Gamma <= 0.05
        assert abs(x.eps_d + x.U / 2) <= 0.02
        assert x.n_keep in sweep.NKEEP_CHOICES
        assert x.Lambda == 2.0 and x.n_iterations == 50
    assert len({x.n_keep for x in a}) == 4


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        share = sweep.rank_share(sweep.sweep_instances(), rank, world)
        mine = [x.index for x in share]
        allv = [None] * world
        dist.all_gather_object(allv, mine)   # check only: the sweep itself exchanges nothing
        q.put((rank, mine, allv, sum(x.cost() for x in share)))
    finally:
        dist.destroy_process_group()


def test_two_rank_split_covers_every_instance_once():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    (_, m0, all0, c0), (_, m1, all1, c1) = out
    assert all0 == all1 == [m0, m1]
    assert sorted(m0 + m1) == list(range(64)) and not set(m0) & set(m1)
    total = c0 + c1
    assert abs(c0 - c1) <= max(x.cost() for x in sweep.sweep_instances()) and total > 0


def test_memory_concurrency_fits_the_largest_instances():
    xs = sweep.sweep_instances()
    big = max(x.device_bytes() for x in xs)
    assert sweep.memory_concurrency(xs, free_bytes=170e9, limit=8) <= int(0.85 * 170e9 // big) + 1
    assert sweep.memory_concurrency(xs, free_bytes=1e9, limit=8) == 1
    small = [x for x in xs if x.n_keep == 512]
    assert sweep.memory_concurrency(small, free_bytes=170e9, limit=8) == 8
