"""Autotuner for the tile shapes of the mixed-precision dense solve.

Two shapes of the packed-panel triangular solves are tunable per handle
(``grim_set_tuning``): the output-tile width of their tensor-core GEMMs (64 or 128
right-hand-side columns per CTA) and the row block of the packed panels (128, 256 or
512).  Which pair is fastest depends on N, the number of right-hand sides and the GPU, so
the tuner times a complete mixed solve (partial pivoting, refinement to the backward-error
target) of the seeded airfoil's linear-Galerkin TM system of the requested size for every
pair and keeps the fastest, per (device, N bucket, right-hand-side bucket), in a
JSON cache (``GRIM_TUNING_CACHE``, default ``~/.cache/grim_20261007_b200/tuning.json``).
``apply`` sets a handle from the cache before a solve; without an entry the library's
built-in rule applies.  With ``GRIM_AUTOTUNE=1`` a missing entry is tuned on first use.
"""
from __future__ import annotations

import itertools
import json
import os
import threading

from . import _lib

CANDIDATES = {'solve_bn': (64, 128), 'gs_block': (128, 256, 512)}
_lock = threading.Lock()
_table = None


def cache_path():
    return os.environ.get('GRIM_TUNING_CACHE') or os.path.join(os.path.expanduser('~'), '.cache',
                                                                'grim_20261007_b200', 'tuning.json')


def bucket(n, nrhs):
    """Cache key parts: N rounded up to a multiple of 512, right-hand sides to a power of two (>= 16)."""
    nb = max(512, -(-int(n) // 512) * 512)
    rb = 16
    while rb < int(nrhs):
        rb *= 2
    return nb, rb


def _key(device_name, n, nrhs):
    nb, rb = bucket(n, nrhs)
    return f'{device_name}|n{nb}|r{rb}'


def _load():
    global _table
    if _table is None:
        try:
            with open(cache_path()) as f:
                _table = json.load(f)
        except (OSError, ValueError):
            _table = {}
    return _table


def _store(key, entry):
    table = _load()
    table[key] = entry
    path = cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + '.tmp'
        with open(tmp, 'w') as f:
            json.dump(table, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass  # an unwritable cache only costs re-tuning in the next process


def lookup(device_name, n, nrhs):
    with _lock:
        return _load().get(_key(device_name, n, nrhs))


def set_handle(ctx, solve_bn=0, gs_block=0):
    _lib.check(ctx.lib.grim_set_tuning(ctx.h, _lib.TUNE_SOLVE_BN, int(solve_bn)), 'grim_set_tuning')
    _lib.check(ctx.lib.grim_set_tuning(ctx.h, _lib.TUNE_GS_BLOCK, int(gs_block)), 'grim_set_tuning')


def apply(ctx, n, nrhs):
    """Set the handle's tile shapes for an (n, nrhs) mixed solve from the cache (built-in
    rule when there is no entry; tuned now when GRIM_AUTOTUNE=1)."""
    entry = lookup(ctx.device_name, n, nrhs)
    if entry is None and os.environ.get('GRIM_AUTOTUNE') == '1':
        entry = tune_dense(n, nrhs, ctx=ctx)
    choice = (entry or {}).get('choice', {})
    set_handle(ctx, choice.get('solve_bn', 0), choice.get('gs_block', 0))
    return choice


def tune_dense(n, nrhs, ctx=None, reps=2, seed=0):
    """Time a mixed solve of a seeded n-panel airfoil with nrhs angles for every candidate
    pair; store and return {'choice': {...}, 'timings_ms': {...}}."""
    import numpy as np
    import torch

    from . import synthetic as S
    from .device import context
    from .twod import operators as ops
    from .twod.galerkin import GalerkinBody
    ctx = ctx or context()
    n = int(n) + (int(n) & 1)
    v, k, _f, _t = S.airfoil_case(seed, n)
    body = GalerkinBody([v], ctx=ctx)
    ang = torch.as_tensor(np.arange(int(nrhs)) * (360.0 / int(nrhs)), device='cuda')
    z32 = ops.fill(body, k, 'TM', complex64=True, ctx=ctx)
    b0 = ops.rhs(body, k, 'TM', ang, ctx=ctx)
    timings = {}
    for bn, gb in itertools.product(CANDIDATES['solve_bn'], CANDIDATES['gs_block']):
        set_handle(ctx, bn, gb)
        times = []
        for r in range(reps + 1):
            b = b0.clone()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            ops.solve_inplace(None, b, 'mixed', tol=ops.MIXED_RCS_TOL, z32=z32, ctx=ctx, stop='berr',
                              tuned=False, pivot=body.pivot)
            e1.record()
            torch.cuda.synchronize()
            if r:  # the first run allocates the workspaces
                times.append(e0.elapsed_time(e1))
        timings[f'solve_bn={bn},gs_block={gb}'] = min(times)
    best = min(timings, key=timings.get)
    choice = dict(item.split('=') for item in best.split(','))
    choice = {key: int(val) for key, val in choice.items()}
    set_handle(ctx, choice['solve_bn'], choice['gs_block'])
    entry = {'choice': choice, 'timings_ms': timings, 'n': n, 'nrhs': int(nrhs)}
    with _lock:
        _store(_key(ctx.device_name, n, nrhs), entry)
    return entry
