"""Benchmark: RCS solves/s at N=2048 (mixed vs FP64 GPU), the 2-D airfoil workload.

Workload (one "step"): the seeded NACA 00tt airfoil (chord 1 m, tt ~ U[8,15] %, cosine
spacing, blunt trailing edge closed by two base elements) with N = 2048 elements at
lambda/10 on average (~30 GHz), 720 monostatic angles (0..359.5 deg by 0.5), both
polarisations (TM = HH, TE = VV) in the reference's own linear-Galerkin combined-field
formulation: two solves per step, each = fill + partial-pivoting LU + 720-RHS solve +
refinement + far field.  The headline arm is the mixed-precision path (complex64 fill and
LU, FP64 refinement); the FP64 GPU path is timed on the same inputs for the ratio; both
are compared with the reference solver's own amplitudes for this airfoil (the committed
fixture tests/golden/ref_airfoil.npz).  ``--formulation pulse`` times the pulse-basis
point-matched EFIE / MFIE instead.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl grim|reference]

Multi-GPU (torchrun): every rank solves its own seeded airfoil (independent units, no
data-path collective: weak scaling); the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = 'RCS solves/s at N=2048 (mixed vs FP64 GPU, <=0.05 dB); p50/p99 serve latency'
UNIT = 'solves/s'


# DRAM bytes (read + write) of one captured launch of the tensor-core kernels, from one ncu
# capture of each kernel on the N = 2048 airfoil, with that launch's algorithmic flops; a
# launch's traffic is scaled from it by its flops.
NCU_TRAFFIC = {
    'k_tc_gemm<128>': (8.833024e6, 8.0 * 512 * 720 * 256),
    'k_oz_gemm': (454.434816e6 + 23.171584e6, 8.0 * 2048 * 2048 * 720),
}


def _peaks():
    try:
        with open(os.path.join(ROOT, 'MEASURED_PEAKS.json')) as f:
            p = json.load(f)
        return float(p['hbm_gbs']), float(p['bf16_tflops']), 'measured'
    except Exception:
        return 6650.0, 1590.0, 'fallback'


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    FIELDS = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
              'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
              'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix='.csv')
            os.close(fd)
            self.proc = subprocess.Popen(['nvidia-smi', f'--id={self.index}', f'--query-gpu={self.FIELDS}',
                                          '--format=csv,noheader,nounits', '-lms', '200'],
                                         stdout=open(self.path, 'w'), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        out = {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': [], 'samples': 0}
        if not self.path or not os.path.exists(self.path):
            return out
        sm, mx, reasons = [], [], set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for line in open(self.path):
            parts = [p.strip() for p in line.split(',')]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == 'active':
                    reasons.add(nm)
        os.unlink(self.path)
        if sm:
            out.update(sm_mhz=statistics.median(sm), sm_max_mhz=max(mx), reasons=sorted(reasons), samples=len(sm))
        return out


def profile_step(ctxs, fn):
    """Run fn once with libgrimgpu's per-launch event profiling on every context in ctxs;
    returns {kernel: stats} summed over them."""
    import ctypes
    import torch
    torch.cuda.synchronize()
    for c in ctxs:
        c.lib.grim_profile_enable(c.h, 1)
    fn()
    torch.cuda.synchronize()
    merged = {}
    for c in ctxs:
        buf = ctypes.create_string_buffer(1 << 16)
        c.lib.grim_profile_report(c.h, buf, len(buf))
        c.lib.grim_profile_enable(c.h, 0)
        for name, v in json.loads(buf.value.decode()).items():
            m = merged.setdefault(name, {'launches': 0, 'ms': 0.0, 'flops': 0.0, 'bytes': 0.0})
            for key in m:
                m[key] += v[key]
    return merged


def run_serving(args):
    """Seeded Poisson stream of mixed requests at ~80% of the measured service rate."""
    from grim_20261007_b200.serving import ServingEngine, synthetic_stream
    reqs, gaps = synthetic_stream(args.seed + 17, args.serving_requests, nmax=8192, angle_max=720)
    probe, _ = synthetic_stream(args.seed + 17, args.serving_requests, nmax=8192, angle_max=720)
    eng = ServingEngine(slots=1)
    t0 = time.perf_counter()
    for r in probe[: max(4, len(probe) // 4)]:
        eng.submit(r).result()
    service = (time.perf_counter() - t0) / max(4, len(probe) // 4)
    eng.close()
    rate = 0.8 / service  # requests per second at ~80% load of one slot's service rate
    eng = ServingEngine(slots=4)
    futs = []
    t0 = time.perf_counter()
    due = 0.0
    for r, g in zip(reqs, gaps):
        due += g / rate
        delay = t0 + due - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        futs.append(eng.submit(r))
    for f in futs:
        f.result()
    st = eng.stats()
    eng.close()
    st.update(requests=len(reqs), arrival_rate_per_s=rate, mean_service_s_single_slot=service,
              mix='2-D superellipse/airfoil N~U[64,8192] (TM/TE), BoR ogives |m|<=U{8..40}, 1-720 angles, '
                  '30% repeat geometries, mixed precision')
    return st


def run_bor(args):
    """Body-of-revolution ogive: 400 generatrix segments (--bor-segments), |m| <= 40, 361 aspects, VV/HH, in
    the reference's default formulation for a closed body (CFIE, alpha = 0.5)."""
    import torch
    from grim_20261007_b200 import synthetic as S
    from grim_20261007_b200.bor.solver import solve_bor_device
    gen, length, half = S.ogive_case(args.seed, n=args.bor_segments)
    k = 25.0 / max(1e-9, float(np.max(gen[:, 0])))  # k rho_max = 25 (the reference's |m| <= 40 converges)
    th = np.arange(361) * 0.5
    out = {'length_m': length, 'half_angle_deg': half, 'k': k, 'segments': args.bor_segments, 'modes': 81, 'aspects': 361,
           'formulation': 'cfie'}
    res = {}
    for prec in ('double', 'mixed'):
        solve_bor_device(gen, k, th, 40, precision=prec, alpha=0.5)  # warm-up at the timed size (workspaces)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        F, tele = solve_bor_device(gen, k, th, 40, precision=prec, alpha=0.5)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        res[prec] = F
        out[prec] = {'seconds': dt, 'solves_per_s': 1.0 / dt, 'refinement_steps': tele['refinement_steps'],
                     'fp64_fallback_modes': tele.get('fp64_fallback_modes', 0),
                     'fp64_fallback_mode_list': tele.get('fp64_fallback_mode_list', []),
                     'max_backward_error': tele.get('max_backward_error'),
                     'max_relative_residual': tele.get('max_relative_residual'),
                     'max_cond': tele.get('max_cond'),
                     'gate_refined_modes': tele.get('gate_refined_modes', []),
                     'stage_seconds': tele.get('stage_seconds')}
    s64 = 4 * np.pi * np.abs(res['double']) ** 2
    s32 = 4 * np.pi * np.abs(res['mixed']) ** 2
    db = 10 * np.log10(np.maximum(s64, 1e-30))
    mask = db > db.max() - 40
    out['max_db_error_mixed_vs_fp64'] = float(np.max(np.abs(10 * np.log10(s32[mask] / s64[mask]))))
    out['k_rho_max'] = float(k * np.max(gen[:, 0]))
    return out


def run_far_block(args):
    """Galerkin far-field element-pair blocks (boundary B2, the reference's dominant fill
    pass): a 1024 x 1024 tile of linear elements on the seeded airfoil (every pair farther
    than 3 element lengths, 6 x 6 Gauss points, S, K and mirrored K), on the GPU
    (device-resident inputs: CUDA events; host buffers through ghost_far_block: wall
    clock) and, where it was built, the reference's own far.c on one host core over a
    bounded sample of rows."""
    import ctypes
    import torch
    from grim_20261007_b200 import synthetic as S
    from grim_20261007_b200.device import context
    from grim_20261007_b200.twod.farblock import KernelTable, far_block
    v, _k, _f, _t = S.airfoil_case(args.seed, 1024)
    a, b = v, np.roll(v, -1, axis=0)
    x, w = np.polynomial.legendre.leggauss(6)
    sfrac = (x + 1) / 2
    pts = np.ascontiguousarray(a[:, None, :] * (1 - sfrac)[None, :, None] + b[:, None, :] * sfrac[None, :, None])
    tan = b - a
    length = np.linalg.norm(tan, axis=1)
    normal = np.ascontiguousarray(np.stack([tan[:, 1], -tan[:, 0]], -1) / length[:, None])
    qw = np.ascontiguousarray(w * 0.5)
    phi = np.ascontiguousarray(np.stack([(1 - x) / 2, (1 + x) / 2], -1))
    cent = (a + b) / 2
    far = np.ascontiguousarray((np.linalg.norm(cent[:, None] - cent[None], axis=-1) > 3 * length.max())
                               .astype(np.uint8))
    k = 2 * np.pi / (10 * np.median(length))  # 10 elements per wavelength
    table = KernelTable(k, 1.2)  # chord 1 m: every distance lies inside the table
    mb = nb = len(v)
    pairs = int(far.sum())
    ctx = context()
    dev = {key: torch.as_tensor(val, device='cuda') for key, val in
           dict(o=pts, s=pts, qw=qw, phi=phi, on=normal, sn=normal, far=far).items()}
    db = torch.as_tensor(table.bounds, device='cuda')
    dc = torch.as_tensor(table.normalized_power.view(np.float64).ravel(), device='cuda')
    accs = [torch.zeros((4, mb, nb), dtype=torch.complex128, device='cuda') for _ in range(3)]
    ptrs = [ctypes.c_void_p(dev[key].data_ptr()) for key in ('o', 's', 'qw', 'phi', 'on', 'sn', 'far')]

    def run_dev():
        for acc in accs:
            acc.zero_()
        return ctx.lib.grim_far_block(ctx.h, mb, nb, 6, 2, *ptrs, 1, 1, 1, 1, k, 0.0, len(table.bounds) - 1,
                                      ctypes.c_void_p(db.data_ptr()), table.normalized_power.shape[1] - 1,
                                      ctypes.c_void_p(dc.data_ptr()), *(ctypes.c_void_p(t.data_ptr()) for t in accs))
    assert run_dev() == 0
    times = []
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        assert run_dev() == 0
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1) / 1e3)
    t_dev = float(np.median(times))
    far_block(table, k, pts, pts, qw, phi, normal, normal, far, 1, True, True, True)
    t0 = time.perf_counter()
    host = far_block(table, k, pts, pts, qw, phi, normal, normal, far, 1, True, True, True)
    t_host = time.perf_counter() - t0
    # algorithmic FP64 operations of one pair (width 2, q = 6, inside the table): per point pair
    # 6 (distance) + 3 (interval coordinate) + 96 (two degree-12 complex Horner chains) + 6 (K
    # projection) + 18 (S, K partial sums) + 16 (mirrored K), per observation point 52
    flops_pair = 36 * 145 + 6 * 52
    out = {'tile': f'{mb} x {nb} linear elements, 6 x 6 points, S + K + mirrored K', 'far_pairs': pairs,
           'kernel_table_intervals': len(table.bounds) - 1,
           'gpu_device_seconds': t_dev, 'gpu_pairs_per_s': pairs / t_dev,
           'roofline': {'bound': 'fp64 pipe (separately rounded multiply and add, no FMA, for bitwise parity)',
                        'flops_per_pair': flops_pair, 'achieved_tflops': pairs * flops_pair / t_dev / 1e12,
                        'peak_tflops_nominal_fp64_no_fma': 20.0,
                        'frac': pairs * flops_pair / t_dev / 1e12 / 20.0},
           'gpu_host_buffers_seconds': t_host, 'gpu_host_buffers_pairs_per_s': pairs / t_host}
    ref_lib = os.path.join(ROOT, 'oracle', '_ref', 'libghost_far_ref.so')
    if os.path.exists(ref_lib):
        lib = ctypes.CDLL(ref_lib)
        fun = lib.ghost_far_block
        p = ctypes.c_void_p
        fun.argtypes = [ctypes.c_int64, ctypes.c_int64, ctypes.c_int, ctypes.c_int] + [p] * 7 + [ctypes.c_int] * 4 + \
            [ctypes.c_double] * 2 + [ctypes.c_int, p, ctypes.c_int, p, p, p, p]
        fun.restype = ctypes.c_int
        rows = 64
        sub = [np.zeros((4, rows, nb), complex) for _ in range(3)]
        pw = np.ascontiguousarray(table.normalized_power)
        t0 = time.perf_counter()
        st = fun(rows, nb, 6, 2, pts.ctypes.data, pts.ctypes.data, qw.ctypes.data, phi.ctypes.data,
                 normal.ctypes.data, normal.ctypes.data, far.ctypes.data, 1, 1, 1, 1, k, 0.0, len(table.bounds) - 1,
                 table.bounds.ctypes.data, pw.shape[1] - 1, pw.ctypes.data, *(a_.ctypes.data for a_ in sub))
        t_ref = time.perf_counter() - t0
        sample_pairs = int(far[:rows].sum())
        same = st == 0 and all(np.array_equal(h_[:, :rows], s_) for h_, s_ in zip(host, sub))
        out.update(reference_cpu_pairs_per_s=sample_pairs / t_ref, reference_cpu_cores=1,
                   reference_sample=f'first {rows} observation elements ({sample_pairs} far pairs)',
                   gpu_vs_reference_cpu=(pairs / t_host) / (sample_pairs / t_ref),
                   bitwise_equal_to_reference_on_sample=bool(same))
    return out


def run_sweep(args, rank=0, world=1):
    """Frequency sweep on the seeded airfoil: 256 frequencies log-spaced over 20:1, N = 10 panels
    per wavelength (uneven sizes), 181 angles, TM, mixed precision.  Timed twice: every system
    on the device worker pool with its own factorization (largest first), and the grouped
    path (one grouped LU of all systems, replayed as a CUDA graph, then solves on the pool),
    which is the reported sweep time; a spread sample of 8 frequencies is re-solved in FP64.
    With several ranks the frequencies are split by the LPT rule (no data-path collective)
    and the sweep time is the maximum over ranks."""
    import torch
    from grim_20261007_b200 import synthetic as S
    from grim_20261007_b200.device import run_pool
    from grim_20261007_b200.sharding import max_over_ranks, my_units
    from grim_20261007_b200.twod import galerkin, geometry as geo, operators as ops
    from grim_20261007_b200.twod.solver import sweep_workers
    cases, thick = S.airfoil_sweep_case(args.seed + 3, args.sweep)
    ang = np.arange(181) * 1.0
    ang_dev = torch.as_tensor(ang, device='cuda')
    all_n = [len(v) for v, _k, _f in cases]
    costs_all = [float(n) ** 3 + 181.0 * n * n for n in all_n]
    mine = my_units(costs_all, rank, world)
    if args.formulation == 'galerkin':
        bodies = {i: galerkin.GalerkinBody([cases[i][0]]) for i in mine}
    else:
        bodies = {i: ops.DeviceBody(geo.panel_geometry([cases[i][0]]), None) for i in mine}
    ns = [bodies[i].n for i in mine]

    def jobs(prec, idx):
        return [(lambda i=i: ops.monostatic_solve(bodies[i], cases[i][1], ang, 'TM', precision=prec,
                                                  angles_dev=ang_dev)) for i in idx]

    idx = mine
    costs = [costs_all[i] for i in idx]
    workers = sweep_workers(len(idx))
    big = sorted(idx, key=lambda i: -costs_all[i])[: 2 * workers]
    run_pool(jobs('mixed', big), workers=workers)  # warm-up: every worker's workspaces at their largest size
    torch.cuda.synchronize()

    def timed(fn):
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        out = fn()
        e1.record()
        torch.cuda.synchronize()
        return out, max_over_ranks(e0.elapsed_time(e1) / 1e3, device='cuda')

    # per system on the worker pool (each system's own factorization chain)
    outs_pool, sec_pool = timed(lambda: run_pool(jobs('mixed', idx), workers=workers, costs=costs))
    # grouped: one captured launch sequence factors every system, then solves on the pool
    # (the first call captures the graph; the timed one replays it)
    grouped = lambda: ops.monostatic_solves_grouped([bodies[i] for i in idx], [cases[i][1] for i in idx], ang, 'TM',
                                                    precision='mixed', angles_dev=ang_dev, workers=workers)
    grouped()
    torch.cuda.synchronize()
    outs, sec = timed(grouped)
    pos = {i: p for p, i in enumerate(idx)}
    sample = [idx[int(round(x))] for x in np.linspace(0, len(idx) - 1, min(8, len(idx)))]
    ref = run_pool(jobs('double', sample), workers=workers)
    err = 0.0
    for i, r in zip(sample, ref):
        s64 = ops.sigma_2d(r['amplitude'].cpu().numpy(), cases[i][1])
        s32 = ops.sigma_2d(outs[pos[i]]['amplitude'].cpu().numpy(), cases[i][1])
        db = ops.sigma_db(s64)
        mask = db > db.max() - 40
        err = max(err, float(np.max(np.abs(10 * np.log10(s32[mask] / s64[mask])))))
    return {'systems': len(cases), 'band': '20:1', 'frequency_ghz': [cases[0][2] / 1e9, cases[-1][2] / 1e9],
            'n_min': min(all_n), 'n_max': max(all_n), 'angles': 181, 'polarization': 'TM', 'thickness': thick,
            'ranks': world, 'workers_per_rank': workers,
            'path': ('per-system partial-pivoting solves on the device worker pool (linear Galerkin)'
                     if args.formulation == 'galerkin' else 'grouped LU (one CUDA graph) + pooled solves'),
            'seconds': sec, 'solves_per_s': len(cases) / sec,
            'per_system_pool': {'seconds': sec_pool, 'solves_per_s': len(cases) / sec_pool},
            'fp64_fallbacks': sum(1 for o in outs if o['telemetry'].get('fp64_fallback')),
            'max_db_error_vs_fp64_sampled': err, 'sampled_frequencies': len(sample)}


def reference_far_block_fn():
    """The reference's own far pass (``twod/assembly/native/far.c`` compiled from its sources
    into oracle/_ref) as ``fn(mb, nb, q, obs_pts, src_pts, qw, phi, obs_norm, src_norm, far,
    table)``, or None where it was not built."""
    import ctypes
    path = os.path.join(ROOT, 'oracle', '_ref', 'libghost_far_ref.so')
    if not os.path.exists(path):
        return None
    lib = ctypes.CDLL(path)
    fun = lib.ghost_far_block
    p = ctypes.c_void_p
    fun.argtypes = [ctypes.c_int64, ctypes.c_int64, ctypes.c_int, ctypes.c_int] + [p] * 7 + [ctypes.c_int] * 4 + \
        [ctypes.c_double] * 2 + [ctypes.c_int, p, ctypes.c_int, p, p, p, p]
    fun.restype = ctypes.c_int

    def run(mb, nb, q, obs_pts, src_pts, qw, phi, obs_norm, src_norm, far, table):
        accs = [np.zeros((4, mb, nb), complex) for _ in range(3)]
        pw = np.ascontiguousarray(table.normalized_power)
        st = fun(mb, nb, q, 2, obs_pts.ctypes.data, src_pts.ctypes.data, qw.ctypes.data, phi.ctypes.data,
                 obs_norm.ctypes.data, src_norm.ctypes.data, far.ctypes.data, 1, 1, 1, 1, table.k, 0.0,
                 len(table.bounds) - 1, table.bounds.ctypes.data, pw.shape[1] - 1, pw.ctypes.data,
                 *(a_.ctypes.data for a_ in accs))
        if st not in (0, 2):
            raise RuntimeError(f'ghost_far_block returned {st}')
        return accs
    return run


def cpu_solve_seconds(v, k, ang, rows, near=True):
    """One solve of the workload by the CPU port (oracle/galerkin_cpu.py) on this process:
    the far pass of element rows ``rows`` (None: all), the near pass, LU / solve / loads /
    far field at full size."""
    from oracle import galerkin_cpu as GC
    fn, table = reference_far_pass(v, k)
    return GC.time_solve(v, k, ang, rows, far_block_fn=fn, table=table, near=near)


_FAR_PASS = {}


def reference_far_pass(v, k):
    """(compiled far-block function, its kernel table) for the contour v, or (None, None);
    built once per process and wavenumber, as the reference keeps its table per solve."""
    key = (float(k), np.asarray(v).tobytes())
    if key not in _FAR_PASS:
        fn = reference_far_block_fn()
        table = None
        if fn is not None:
            from grim_20261007_b200.twod.farblock import KernelTable
            table = KernelTable(k, 1.2 * float(np.max(np.ptp(v, axis=0))) * math.sqrt(2.0))
            table.k = k
        _FAR_PASS.clear()
        _FAR_PASS[key] = (fn, table)
    return _FAR_PASS[key]


def cpu_baseline_sample(args, v, k, ang):
    """The CPU port timed on one host core: one full TM solve of the workload (every
    element row's far pass, every near pair, LAPACK LU and solve, loads, far field)."""
    sec, parts = cpu_solve_seconds(v, k, ang, None)
    return {'value': 1.0 / sec, 'unit': UNIT, 'cores': 1, 'kind': 'port',
            'sample': f'one full TM solve of the workload (N={args.n}, {len(ang)} angles): far pairs by the '
                      'reference\'s own compiled far.c (upper triangle, mirrored), near pairs by the oracle\'s '
                      'Galerkin rules batched in NumPy as the reference batches them, LAPACK LU and solve',
            'parts': parts}


def workload(seed, n, nang):
    from grim_20261007_b200 import synthetic as S
    v, k, f, t = S.airfoil_case(seed, n)
    ang = np.arange(nang) * (360.0 / nang)
    return v, k, f, t, ang


def _ref_far_worker(payload):
    """One spawned process of the reference arm: the far pass of its element rows."""
    v, k, rows = payload
    sys.path.insert(0, ROOT)
    from oracle import galerkin_cpu as GC
    fn, table = reference_far_pass(v, k)
    t0 = time.perf_counter()
    if fn is not None:
        GC.far_all_compiled(v, k, fn, table, rows)
    else:
        GC.far_rows_numpy(v, k, rows)
    return time.perf_counter() - t0


def run_reference_arm(args, rank, world):
    """The reference's CPU path for this workload on all host cores (rank 0 only): the CPU
    port of oracle/galerkin_cpu.py -- the far pass by the reference's own compiled far.c,
    its element rows split over spawned processes, the batched near pass in the main process
    meanwhile, then LAPACK LU and the 720-angle solve on all cores; one step = TM + TE."""
    if rank != 0:
        return
    import concurrent.futures as cf
    import multiprocessing as mp
    from oracle import galerkin_cpu as GC
    cores = os.cpu_count() or 1
    v, k, f, t, ang = workload(args.seed, args.n, args.angles)
    chunks = [np.arange(i, args.n, cores) for i in range(cores)]
    ctx = mp.get_context('spawn')

    def one_solve(pool):
        t0 = time.perf_counter()
        futs = [pool.submit(_ref_far_worker, (v, k, c)) for c in chunks]
        GC.near_all(v, k)
        for fu in futs:
            fu.result()
        _total, parts = cpu_solve_seconds(v, k, ang, [], near=False)   # LU, solve, loads, far field
        return time.perf_counter() - t0 - parts['far_fill_s']

    with cf.ProcessPoolExecutor(max_workers=cores, mp_context=ctx) as pool:
        for _ in range(args.warmup):
            one_solve(pool)
        secs = [one_solve(pool) + one_solve(pool) for _ in range(args.steps)]
    dt = float(np.sum(secs))
    value = 2 * args.steps / dt
    line = {
        'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': world, 'steps': args.steps, 'warmup': args.warmup,
        'ms_per_step': dt / args.steps * 1e3, 'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
        'dtype': 'f64', 'data': 'synthetic (seeded NACA 00tt airfoil)', 'impl': 'reference',
        'config': {'workload': f'2-D airfoil N={args.n}, {args.angles} angles, TM+TE, linear-Galerkin combined '
                               'formulation, FP64 CPU', 'n_elements': args.n, 'angles': args.angles, 'seed': args.seed},
        'cpu_baseline': {'value': value, 'unit': UNIT, 'cores': cores, 'kind': 'port',
                         'sample': f'full TM + TE solves per step: the far pass by the reference\'s compiled far.c '
                                   f'over {cores} spawned processes, the oracle\'s batched near pass, LAPACK LU and '
                                   'solve on all cores'},
        'e2e': {'value': value, 'unit': UNIT, 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
    }
    print(json.dumps(line), flush=True)


def reference_parity(args, rank, k, amp64, amp32):
    """Max dB and relative amplitude differences of both arms from the reference solver's
    own amplitudes (tests/golden/ref_airfoil.npz: its solve_monostatic_rcs_2d_single_
    polarization on synthetic.airfoil_case(0, n), 720 angles) where sigma is within 40 dB
    of its peak; None when this rank's workload is not the fixture's."""
    path = os.path.join(ROOT, 'tests', 'golden', 'ref_airfoil.npz')
    if not os.path.exists(path) or args.seed + rank != 0 or args.angles != 720:
        return None
    g = np.load(path)
    if args.n not in [int(x) for x in g['sizes']] or abs(float(g[f'n{args.n}_k']) - k) > 1e-12 * k:
        return None
    out = {'reference': 'GHOST solve_monostatic_rcs_2d_single_polarization (its own stored amplitudes)'}
    for pol in ('TM', 'TE'):
        ref = g[f'n{args.n}_amp_{pol}']
        db_ref = 10 * np.log10(np.abs(ref) ** 2)
        mask = db_ref > db_ref.max() - 40
        for arm, amp in (('fp64', amp64[pol]), ('mixed', amp32[pol])):
            db = 10 * np.log10(np.abs(amp) ** 2)
            out[f'{pol}_{arm}_max_db'] = float(np.max(np.abs(db - db_ref)[mask]))
            out[f'{pol}_{arm}_max_rel_amp'] = float(np.max(np.abs(amp - ref)) / np.max(np.abs(ref)))
    return out


def own_gemm_rates():
    """Large square GEMMs through this build's own tensor-core kernels, as the compute
    denominators of the solve arms (no library GEMM is timed): the FP64 DMMA kernel
    (complex128 residual R = B - A X at n = nrhs = 4096, 550 GFLOP) and the split-TF32
    tcgen05 kernel (complex64 C -= A B at 8192^3, 4.4 TFLOP algorithmic 8 M N K), CUDA
    events, one warm-up call, median of three."""
    import torch
    from grim_20261007_b200.device import context, ptr
    ctx = context()
    out = {}
    n = 4096
    g = torch.Generator(device='cuda').manual_seed(0)
    a = torch.randn((n, n), dtype=torch.complex128, device='cuda', generator=g)
    x = torch.randn((n, n), dtype=torch.complex128, device='cuda', generator=g)
    b = torch.randn((n, n), dtype=torch.complex128, device='cuda', generator=g)
    r = torch.empty_like(b)

    def timed(fn, reps=3):
        fn()
        torch.cuda.synchronize()
        ms = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        return float(np.median(ms))

    ms = timed(lambda: ctx.lib.grim_residual(ctx.h, n, n, ptr(a), n, 0, ptr(x), n, ptr(b), n, ptr(r), n, 0))
    out['fp64_dmma'] = {'kernel': 'k_gemm_dmma', 'm_n_k': [n, n, n], 'ms': ms, 'tflops': 8.0 * n ** 3 / (ms * 1e-3) / 1e12,
                        'nominal_fp64_tensor_tflops': 40.0}
    del a, x, b, r
    m = 8192
    a = torch.randn((m, m), dtype=torch.complex64, device='cuda', generator=g)
    bb = torch.randn((m, m), dtype=torch.complex64, device='cuda', generator=g)
    c = torch.zeros((m, m), dtype=torch.complex64, device='cuda')
    ms = timed(lambda: ctx.lib.grim_cgemm_sub(ctx.h, m, m, m, ptr(a), m, ptr(bb), m, ptr(c), m, 1))
    out['split_tf32'] = {'kernel': 'k_tc_gemm', 'm_n_k': [m, m, m], 'ms': ms,
                         'tflops': 8.0 * m ** 3 / (ms * 1e-3) / 1e12}
    del a, bb, c
    torch.cuda.empty_cache()
    return out


def fp64_roofline(prof64, rates):
    """The FP64 arm's GEMM kernel against the same kernel's large-square rate and the
    nominal FP64 tensor rate."""
    d = prof64.get('k_gemm_dmma')
    if not d or not rates or not rates.get('fp64_dmma', {}).get('tflops'):
        return None
    achieved = d['flops'] / (d['ms'] * 1e-3) / 1e12
    big = rates['fp64_dmma']['tflops']
    return {'kernel': 'k_gemm_dmma', 'launches': d['launches'], 'achieved': achieved, 'unit': 'TFLOP/s',
            'peak_own_large_gemm': big, 'frac_of_own_large_gemm': achieved / big,
            'peak_nominal': 40.0, 'frac_of_nominal': achieved / 40.0,
            'note': 'algorithmic 8 M N K per complex GEMM launch; denominators: the same kernel at 4096^3 '
                    '(measured here) and the nominal FP64 tensor rate (not measured: no library FP64 GEMM is timed)'}


def kernel_roofline(prof):
    """Roofline of the kernel with the largest share of one profiled mixed step."""
    hbm, bf16, src = _peaks()
    dom_name, dom = max(prof.items(), key=lambda kv: kv[1]['ms'])
    step_ms = sum(v['ms'] for v in prof.values())
    base = {'kernel': dom_name, 'launches': dom['launches'], 'avg_launch_ms': dom['ms'] / dom['launches'],
            'share_of_step': dom['ms'] / step_ms, 'peak_source': src, 'traffic': None}
    if 'gepp' in dom_name:
        # the partial-pivoting panel is a chain of 64 dependent column steps per launch:
        # latency-bound; its algorithmic rate is reported against the FP64 / FP32 pipe
        achieved = dom['flops'] / (dom['ms'] * 1e-3) / 1e12
        base.update(bound='latency (column-step chain)', achieved=achieved, peak=bf16, unit='TFLOP/s',
                    frac=achieved / bf16, note='algorithmic 8 m 64^2 / 2 flops per panel; one cluster barrier '
                    'per column; peak = measured dense bf16 tensor rate (the only measured compute peak)')
        return base
    if dom['flops'] > 0:
        achieved = dom['flops'] / (dom['ms'] * 1e-3) / 1e12
        base.update(bound='tensor', achieved=achieved, peak=bf16, unit='TFLOP/s', frac=achieved / bf16)
        if dom_name in NCU_TRAFFIC:
            nbytes, nflops = NCU_TRAFFIC[dom_name]
            base['traffic'] = nbytes * (dom['flops'] / dom['launches']) / nflops
        return base
    achieved = dom['bytes'] / (dom['ms'] * 1e-3) / 1e9
    base.update(bound='hbm', achieved=achieved, peak=hbm, unit='GB/s', frac=achieved / hbm)
    return base


def top_kernels(prof, count=6):
    step_ms = sum(v['ms'] for v in prof.values())
    top = sorted(prof.items(), key=lambda kv: -kv[1]['ms'])[:count]
    return {name: {'ms': round(v['ms'], 4), 'launches': v['launches'], 'share': round(v['ms'] / step_ms, 4)}
            for name, v in top}


def summarize(d, keys):
    if not d:
        return d
    return {k_: d[k_] for k_ in keys if k_ in d}


def summarize_bor(bor):
    if not bor:
        return bor
    out = {k_: bor[k_] for k_ in ('segments', 'modes', 'aspects', 'formulation', 'max_db_error_mixed_vs_fp64')
           if k_ in bor}
    for prec in ('double', 'mixed'):
        if prec in bor:
            out[prec] = {k_: bor[prec][k_] for k_ in ('seconds', 'solves_per_s', 'fp64_fallback_modes',
                                                      'max_backward_error') if k_ in bor[prec]}
    return out


def write_detail(detail):
    """Telemetry, per-kernel profiles and the secondary legs' full records, beside the line."""
    folder = os.path.join(ROOT, 'gpurun_out')
    if not os.path.isdir(folder):
        return None
    path = os.path.join(folder, 'bench_detail.json')
    with open(path, 'w') as fh:
        json.dump(detail, fh, default=str)
    return os.path.relpath(path, ROOT)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=10)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='grim', choices=['grim', 'reference'])
    ap.add_argument('--n', type=int, default=2048)
    ap.add_argument('--angles', type=int, default=720)
    ap.add_argument('--seed', type=int, default=0)
    ap.add_argument('--cpu-sample', type=int, default=1, help='time one full CPU-port solve for cpu_baseline (0 = skip)')
    ap.add_argument('--serving', type=int, default=1, help='run the mixed request stream (p50/p99 latency)')
    ap.add_argument('--serving-requests', type=int, default=32)
    ap.add_argument('--bor', type=int, default=1, help='time the body-of-revolution ogive workload')
    ap.add_argument('--bor-segments', type=int, default=400, help='generatrix segments of the BoR ogive')
    ap.add_argument('--sweep', type=int, default=256, help='frequencies of the airfoil sweep leg (0 = skip)')
    ap.add_argument('--autotune', type=int, default=1, help='tune the solve tile shapes for the workload first')
    ap.add_argument('--far-block', type=int, default=1, help='time the Galerkin far-block pass (boundary B2)')
    ap.add_argument('--formulation', default='galerkin', choices=['galerkin', 'pulse'],
                    help="2-D discretisation: the reference's linear Galerkin (default) or pulse basis")
    args = ap.parse_args()

    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))

    if args.impl == 'reference':
        run_reference_arm(args, rank, world)
        return

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=120))

    from grim_20261007_b200.device import all_contexts, context, run_concurrent
    from grim_20261007_b200.execution import linear_precision
    from grim_20261007_b200.twod import galerkin, geometry as geo, operators as ops
    from grim_20261007_b200.twod.solver import solve_monostatic_rcs_2d
    from grim_20261007_b200 import synthetic as S

    ctx = context()
    v, k, f, thick, ang = workload(args.seed + rank, args.n, args.angles)
    if args.formulation == 'galerkin':
        gal = galerkin.GalerkinBody([v])
        bodies = {'TM': gal, 'TE': gal}
        h2d_body = gal.h2d_bytes
    else:
        geom = geo.panel_geometry([v])
        bodies = {'TM': ops.DeviceBody(geom, None), 'TE': ops.DeviceBody(geom, geo.te_curvature_correction([v]))}
        h2d_body = 2 * geom.nbytes + geom.shape[0] * 8
    ang_dev = torch.as_tensor(ang, device='cuda')
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device='cuda')

    def step(precision):
        # the two polarisations are independent solves: run them on two device workers at once
        pols = ('TM', 'TE')
        res = run_concurrent([
            (lambda p=p: ops.monostatic_solve(bodies[p], k, ang, p, precision=precision, angles_dev=ang_dev))
            for p in pols])
        return dict(zip(pols, res))

    def step_serial(precision):
        # one polarisation after the other on the default context: per-kernel event times
        # are then those of a kernel alone on the GPU (used for the kernel profile only)
        return {p: ops.monostatic_solve(bodies[p], k, ang, p, precision=precision, angles_dev=ang_dev)
                for p in ('TM', 'TE')}

    def launch_count():
        return sum(c.launches for c in all_contexts())

    def barrier():
        if world > 1:
            dist.barrier()

    def timed(precision, steps, warmup):
        for _ in range(warmup):
            step(precision)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        times = []
        launches0 = launch_count()
        last = None
        for _ in range(steps):
            flush.fill_(1.0)  # L2 flush (256 MiB write) outside the event window
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            last = step(precision)
            e1.record()
            times.append((e0, e1))
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        launches = launch_count() - launches0
        ms = [a.elapsed_time(b) for a, b in times]
        return ms, launches, last

    # tile shapes of the mixed solve for this (N, angles): timed candidates, fastest kept (every
    # handle picks it up from the tuner's cache before its solves)
    autotune = None
    if args.autotune:
        from grim_20261007_b200 import tuning
        autotune = tuning.tune_dense(args.n, args.angles, ctx=ctx)

    # FP64 drop-in arm (ratio and accuracy reference)
    ms64, _l64, out64 = timed('double', max(2, args.steps // 2), 1)
    with ClockSampler(local) as clk:
        ms32, launches32, out32 = timed('mixed', args.steps, args.warmup)
    clocks = clk.summary()

    tot = torch.tensor([sum(ms32), sum(ms64)], dtype=torch.float64, device='cuda')
    if world > 1:
        dist.all_reduce(tot, op=dist.ReduceOp.MAX)
    total_ms32, total_ms64 = float(tot[0]), float(tot[1])
    ms_step32 = total_ms32 / args.steps
    ms_step64 = total_ms64 / max(2, args.steps // 2)
    value = 2 * args.steps * world / (total_ms32 / 1e3)
    fp64_value = 2 * world / (ms_step64 / 1e3)

    # accuracy of the mixed arm vs the FP64 arm (dB where sigma is within 40 dB of its peak)
    err_db = {}
    for pol in ('TM', 'TE'):
        a64 = out64[pol]['amplitude'].cpu().numpy()
        a32 = out32[pol]['amplitude'].cpu().numpy()
        s64 = ops.sigma_2d(a64, k)
        s32 = ops.sigma_2d(a32, k)
        db = ops.sigma_db(s64)
        mask = db > db.max() - 40
        err_db[pol] = float(np.max(np.abs(10 * np.log10(s32[mask] / s64[mask]))))
    tele32 = {p: {kk: vv for kk, vv in out32[p]['telemetry'].items() if not hasattr(vv, 'cpu')} for p in ('TM', 'TE')}
    tele64 = {p: {kk: vv for kk, vv in out64[p]['telemetry'].items() if not hasattr(vv, 'cpu')} for p in ('TM', 'TE')}
    berr64 = max(float(out64[p]['telemetry']['backward_error_dev'].max()) for p in ('TM', 'TE'))

    # the same amplitudes against the reference solver's own (its stored complex amplitudes
    # for this airfoil, tests/golden/ref_airfoil.npz), where the workload is the fixture's
    parity = reference_parity(args, rank, k, {p: out64[p]['amplitude'].cpu().numpy() for p in ('TM', 'TE')},
                              {p: out32[p]['amplitude'].cpu().numpy() for p in ('TM', 'TE')})

    # end-to-end through the public API (host geometry in, host amplitudes out)
    snap = S.snapshot_from_polygons([v])
    os.environ['GRIM_2D_FORMULATION'] = args.formulation
    with linear_precision('mixed'):
        solve_monostatic_rcs_2d(snap, [f / 1e9], list(ang), geometry_units='meters', strict_quality_gate=False)
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        e2e_steps = max(2, args.steps // 2)
        for _ in range(e2e_steps):
            solve_monostatic_rcs_2d(snap, [f / 1e9], list(ang), geometry_units='meters', strict_quality_gate=False)
        torch.cuda.synchronize()
        e2e_dt = time.perf_counter() - t0
    e2e_t = torch.tensor([e2e_dt], dtype=torch.float64, device='cuda')
    if world > 1:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_value = 2 * e2e_steps * world / float(e2e_t[0])
    h2d = h2d_body + 2 * len(ang) * 8
    d2h = 2 * len(ang) * 16

    def settle():
        # each leg starts from the same allocator state: cached blocks of the previous leg
        # (the serving engine's factor cache, N up to 8192) are returned to the device
        torch.cuda.synchronize()
        torch.cuda.empty_cache()

    serving = run_serving(args) if (args.serving and rank == 0 and world == 1) else None
    settle()
    bor = run_bor(args) if (args.bor and rank == 0 and world == 1) else None
    settle()
    sweep = run_sweep(args, rank, world) if args.sweep else None
    settle()
    farblk = run_far_block(args) if (args.far_block and rank == 0 and world == 1) else None

    # per-kernel profile of one mixed step, polarisations in turn (CUDA events after every
    # launch on the launching stream, separate from the timed loop)
    n = args.n
    step_serial('mixed')  # the default context's workspaces exist before its profile starts
    step_serial('double')
    prof = profile_step([ctx], lambda: step_serial('mixed'))
    prof64 = profile_step([ctx], lambda: step_serial('double'))
    roofline = kernel_roofline(prof)
    rates = own_gemm_rates() if rank == 0 else None
    roof64 = fp64_roofline(prof64, rates) if rates else None

    cpu_baseline = None
    if rank == 0 and world == 1 and args.cpu_sample > 0:
        cpu_baseline = cpu_baseline_sample(args, v, k, ang)

    if rank == 0:
        detail = {'telemetry_mixed': tele32, 'telemetry_fp64': tele64, 'kernel_profile_mixed': prof,
                  'own_gemm_rates': rates,
                  'kernel_profile_fp64': prof64, 'serving': serving, 'bor_ogive': bor, 'frequency_sweep': sweep,
                  'far_block': farblk, 'autotune': autotune}
        detail_path = write_detail(detail)
        line = {
            'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': world, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': ms_step32, 'higher_is_better': True, 'scaling': 'weak',
            'vs_baseline': None, 'dtype': 'c64+f64', 'data': 'synthetic (seeded NACA 00tt airfoil)',
            'config': {'workload': f'2-D airfoil N={n}, {args.angles} monostatic angles, TM+TE (2 solves/step), '
                                   f'mixed precision, {args.formulation} formulation', 'n_elements': n,
                       'angles': args.angles, 'seed': args.seed, 'frequency_ghz': f / 1e9, 'thickness': thick,
                       'formulation': args.formulation,
                       'l2': 'flushed between steps (256 MiB write outside each step\'s event window)',
                       'parallelism': f'replicas x{world}'},
            'fp64_gpu': {'value': fp64_value, 'ms_per_step': ms_step64, 'max_backward_error': berr64},
            'speedup_vs_fp64': value / fp64_value if fp64_value else None,
            'max_db_error_vs_fp64': err_db,
            'parity_vs_reference': parity,
            'e2e': {'value': e2e_value, 'unit': UNIT, 'h2d_bytes_per_step': int(h2d), 'd2h_bytes_per_step': int(d2h),
                    'path': 'solve_monostatic_rcs_2d (public API), linear_precision("mixed")'},
            'gpu_launches': int(launches32),
            'roofline': roofline,
            'roofline_fp64': roof64,
            'own_gemm_rates': {k_: {'tflops': v_['tflops'], 'kernel': v_['kernel']} for k_, v_ in (rates or {}).items()},
            'top_kernels_mixed': top_kernels(prof),
            'serving': summarize(serving, ('requests', 'completed', 'solves_per_s', 'p50_ms', 'p99_ms', 'cache_hits')),
            'bor_ogive': summarize_bor(bor),
            'frequency_sweep': summarize(sweep, ('systems', 'seconds', 'solves_per_s', 'n_min', 'n_max',
                                                 'max_db_error_vs_fp64_sampled', 'path')),
            'far_block': summarize(farblk, ('gpu_pairs_per_s', 'gpu_host_buffers_pairs_per_s',
                                            'reference_cpu_pairs_per_s', 'bitwise_equal_to_reference_on_sample')),
            'cpu_baseline': cpu_baseline,
            'clocks': clocks,
            'detail_file': detail_path,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == '__main__':
    main()
