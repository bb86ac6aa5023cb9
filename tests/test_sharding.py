"""Work split over ranks (gloo, world size 2, on the CPU): LPT assignment, result gather, max-over-ranks."""
import os
import socket

import numpy as np
import pytest

from grim_20261007_b200.sharding import gather_results, lpt_partition, max_over_ranks, my_units


def test_lpt_partition_covers_every_unit_once_and_balances():
    rng = np.random.default_rng(1)
    costs = (rng.integers(64, 4096, 256).astype(float)) ** 3
    for world in (1, 2, 3, 8):
        owner, load = lpt_partition(costs, world)
        assert sorted(set(owner)) == list(range(min(world, len(costs))))
        parts = [my_units(costs, r, world) for r in range(world)]
        assert sorted(i for p in parts for i in p) == list(range(len(costs)))
        for r in range(world):
            assert abs(load[r] - sum(costs[i] for i in parts[r])) <= 1e-6 * load[r]
        # greedy LPT bound: max load <= mean + max unit
        assert max(load) <= sum(costs) / world + max(costs) + 1e-6
    assert lpt_partition([3.0, 3.0], 4)[0] == [0, 1]  # ties go to the lowest rank


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, costs, out):
    import torch.distributed as dist
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        mine = my_units(costs, rank, world)
        local = [{'unit': i, 'rank': rank, 'value': float(i) ** 2} for i in mine]
        allres = gather_results(local, costs, rank, world)
        t = max_over_ranks(1.5 + rank)
        out.put((rank, [r['unit'] for r in allres], [r['rank'] for r in allres], t))
    finally:
        dist.destroy_process_group()


def test_gather_and_max_over_two_gloo_ranks():
    import torch.multiprocessing as mp
    costs = [float(c) for c in (5, 1, 9, 3, 7, 2, 8, 4)]
    world = 2
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, costs, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    owner, _ = lpt_partition(costs, world)
    for rank, units, ranks, t in got:
        assert units == list(range(len(costs)))   # every rank sees all results, in unit order
        assert ranks == owner                      # each from the rank that owned it
        assert t == 2.5                            # max over ranks of 1.5 + rank
