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


def _failing_worker(rank, world, port, out):
    import torch.distributed as dist
    from grim_20261007_b200.sharding import run_sharded
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        def run_local(idx):
            if rank == 1:
                raise ValueError('planted failure')
            return [i * 10 for i in idx]
        try:
            run_sharded([4.0, 3.0, 2.0, 1.0], run_local)
            out.put((rank, 'no error'))
        except RuntimeError as exc:
            out.put((rank, str(exc)))
    finally:
        dist.destroy_process_group()


def test_run_sharded_reports_a_failed_rank_on_every_rank():
    """A share that raises on one rank: every rank leaves the gather with the same error
    (none waits forever in the collective)."""
    import torch.multiprocessing as mp
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_failing_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for rank in (0, 1):
        assert 'rank(s) 1: ValueError: planted failure' in got[rank]


def _api_worker(rank, world, port, out):
    """One rank of a sharded public 2-D solve whose per-system GPU solve is replaced by a
    host fake that records which rank solved each (frequency, polarisation)."""
    import torch.distributed as dist
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    os.environ['GRIM_SWEEP_WORKERS'] = '1'
    os.environ['GRIM_GROUPED_SWEEP'] = '0'
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        from grim_20261007_b200 import synthetic as S
        from grim_20261007_b200.execution import shard_over_ranks
        from grim_20261007_b200.twod import solver

        class _Ctx:
            device_name = f'fake-{rank}'

        solved = []

        def fake_solve(meshes, f, elevs, pol, precision, abort_event, condition=False):
            solved.append((pol, f))
            samples = [{'frequency_ghz': f, 'theta_inc_deg': e, 'theta_scat_deg': e, 'rcs_linear': 1.0,
                        'rcs_db': 0.0, 'rcs_amp_real': float(rank), 'rcs_amp_imag': 0.0, 'rcs_amp_phase_deg': 0.0,
                        'linear_residual': 1e-15} for e in elevs]
            event = dict(requested='gpu', used='gpu_grim', factorizations=1, rhs_columns=len(elevs), n=8,
                         gpu_device=f'fake-{rank}', precision=precision)
            return dict(samples=samples, residuals=[1e-15] * len(elevs), event=event, n=8, seconds=0.0,
                        condition_est=None)

        solver._solve_frequency = fake_solve
        solver.require_cuda = lambda: None
        solver.context = lambda: _Ctx()
        snap = S.snapshot_from_polygons([S.naca_symmetric(0.12, 40)])
        freqs = [0.5, 1.0, 1.5, 2.0, 2.5]
        with shard_over_ranks():
            res = solver.solve_monostatic_rcs_2d(snap, freqs, [0.0, 90.0], geometry_units='meters')
        rows = [(r['polarization'], r['frequency_ghz'], r['rcs_amp_real']) for r in res['samples']]
        out.put((rank, sorted(solved), rows))
    finally:
        dist.destroy_process_group()


def test_public_2d_solve_splits_its_systems_over_two_gloo_ranks():
    """shard_over_ranks: each rank solves only its LPT share of the 10 (polarisation,
    frequency) systems, and both ranks return the same full result, in frequency order
    (VV then HH for each physical sample)."""
    import torch.multiprocessing as mp
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_api_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(2):
        rank, solved, rows = q.get(timeout=180)
        got[rank] = (solved, rows)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    s0, s1 = set(got[0][0]), set(got[1][0])
    assert not (s0 & s1) and len(s0) + len(s1) == 10 and s0 and s1
    assert got[0][1] == got[1][1]
    freqs = [0.5, 1.0, 1.5, 2.0, 2.5]
    # the reference's co-polarised order: VV then HH for each physical sample
    assert [(p, f) for p, f, _a in got[0][1]] == [(p, f) for f in freqs for _e in (0, 1) for p in ('VV', 'HH')]
    # every system's samples come from the rank that solved it
    pol_of = {'VV': 'TE', 'HH': 'TM'}
    for p, f, a in got[0][1]:
        assert ((pol_of[p], f) in s1) == (a == 1.0)
