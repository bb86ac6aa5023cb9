"""Work split of independent solve units over ranks (one process per GPU).

The path shards without a data-path collective: the units of a request -- the frequencies
of a sweep, the Fourier modes of a body of revolution, the requests of a serving queue --
are independent systems, so each rank solves its own share and only small host results
(far-field vectors, sample records) are gathered at the end.  The assignment is the greedy
longest-processing-time rule on a cost per unit (N^3 + N^2 R for a dense solve), the same
rule the reference's frequency scheduler applies to its worker processes
(``execution/frequency_sweep.py:140`` ``_plan``).

Every rank calls these functions with the same arguments in the same order (they are
collective when a process group is given).
"""
from __future__ import annotations

import heapq

import torch.distributed as dist


def lpt_partition(costs, world):
    """Assign unit i (cost costs[i]) to a rank: largest first, each to the least-loaded rank
    (ties to the lowest rank).  Returns (owner list, per-rank load list); deterministic."""
    world = int(world)
    if world < 1:
        raise ValueError('world must be >= 1')
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world)]
    owner = [0] * len(costs)
    load = [0.0] * world
    for i in order:
        l, r = heapq.heappop(heap)
        owner[i] = r
        load[r] = l + float(costs[i])
        heapq.heappush(heap, (load[r], r))
    return owner, load


def my_units(costs, rank, world):
    """Indices of the units rank ``rank`` solves (in unit order)."""
    owner, _ = lpt_partition(costs, world)
    return [i for i, r in enumerate(owner) if r == rank]


def gather_results(local, costs, rank, world, group=None):
    """Collect every rank's results for its units into one list in unit order.

    ``local`` is the list of this rank's results, in the order of ``my_units``.  With one
    rank (or no process group) it is returned as is.
    """
    if world == 1 or not dist.is_initialized():
        return list(local)
    owner, _ = lpt_partition(costs, world)
    parts = [None] * world
    dist.all_gather_object(parts, list(local), group=group)
    out, taken = [None] * len(costs), [0] * world
    for i, r in enumerate(owner):
        out[i] = parts[r][taken[r]]
        taken[r] += 1
    return out


def max_over_ranks(value, group=None, device=None):
    """Maximum of a float over ranks (the job time of a weak- or strong-scaled step)."""
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device or 'cpu')
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def run_sharded(costs, run_local, group=None):
    """Run units over the ranks of ``group``: this rank calls ``run_local(indices)`` on its
    LPT share (unit indices in unit order; it returns one host result per index, in that
    order), then every rank receives all results in unit order.  Without an initialised
    process group, or with one rank, ``run_local`` gets every unit.  Collective: every rank
    calls it with the same costs.  A rank whose share raised still joins the gather, and
    then every rank raises ``RuntimeError`` naming the failed ranks (no rank is left
    waiting in the collective)."""
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return list(run_local(list(range(len(costs)))))
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    owner, _ = lpt_partition(costs, world)
    mine = [i for i, r in enumerate(owner) if r == rank]
    try:
        local = list(run_local(mine)) if mine else []
        if len(local) != len(mine):
            raise RuntimeError(f'run_local returned {len(local)} results for {len(mine)} units')
        part = (None, local)
    except Exception as exc:  # noqa: BLE001 - reported to every rank below
        part = (f'{type(exc).__name__}: {exc}', [])
    parts = [None] * world
    dist.all_gather_object(parts, part, group=group)
    failed = [(r, p[0]) for r, p in enumerate(parts) if p[0] is not None]
    if failed:
        raise RuntimeError('sharded solve failed on rank(s) ' + '; '.join(f'{r}: {m}' for r, m in failed))
    out, taken = [None] * len(costs), [0] * world
    for i, r in enumerate(owner):
        out[i] = parts[r][1][taken[r]]
        taken[r] += 1
    return out
