"""Continuous-batching RCS request engine on one GPU.

* Requests (2-D closed PEC contours or bodies of revolution) arrive at any time
  (``submit``); each returns a ``concurrent.futures.Future``.
* ``slots`` worker threads each own a libgrimgpu handle and a CUDA stream; a request is
  admitted into a free slot only when its estimated device memory fits in the HBM budget
  next to the requests already running (the reference admits solves by RAM the same way:
  ``twod/solver.py:1474`` ``_estimate_memory_gb``, ``:2382-2398``).  Requests that arrive
  while others run are admitted as soon as a slot and memory free up, so their kernels
  overlap on the device.
* A resident factor cache keeps the system matrix and its LU factors of recent 2-D
  geometries on the device, keyed by (geometry hash, k, polarization, precision); a
  repeat geometry skips the fill and the factorization and only solves its angles.  The
  cache's bytes count against the budget at admission (unpinned entries are evicted to
  make room), and a request admitted as a cache hit pins its entry until it ends.
* ``stats()`` reports completed solves, solves/s and p50/p99 latency (arrival to result).

Results do not depend on what else runs: every kernel's reductions have a fixed order
per problem size, so a request gives the same answer alone and in the mix.
"""
from __future__ import annotations

import collections
import concurrent.futures as cf
import ctypes
import hashlib
import threading
import time

import numpy as np
import torch

from .. import _lib
from ..device import Context, ptr, require_cuda
from ..twod import galerkin, operators as ops


class Request:
    """One RCS solve: kind '2d' (vertices, polarization) or 'bor' (generatrix, both pols)."""

    _ids = 0

    def __init__(self, kind, geometry, k, angles_deg, polarization='TM', precision='mixed', n_modes=None):
        if kind not in ('2d', 'bor'):
            raise ValueError("request kind must be '2d' or 'bor'")
        Request._ids += 1
        self.id = Request._ids
        self.kind = kind
        self.geometry = np.ascontiguousarray(np.asarray(geometry, dtype=np.float64))
        self.k = float(k)
        self.angles = np.ascontiguousarray(np.asarray(angles_deg, dtype=np.float64).reshape(-1))
        self.pol = ops.canonical_pol(polarization) if kind == '2d' else 'VV+HH'
        self.precision = precision
        self.n_modes = n_modes
        self.pinned = None  # cache key this request pinned at admission
        self.arrival = None
        self.started = None
        self.finished = None
        self.cache_hit = False

    @property
    def n(self):
        return len(self.geometry) if self.kind == '2d' else 2 * len(self.geometry)

    def cache_key(self):
        h = hashlib.sha256(self.geometry.tobytes()).hexdigest()[:24]
        return (self.kind, h, round(self.k, 12), self.pol, self.precision)

    def estimate_bytes(self, cached=False):
        """Device memory while running (matrix, factors, right-hand sides, workspace)."""
        r = max(1, len(self.angles))
        if self.kind == '2d':
            esz = 8 if self.precision == 'mixed' else 16
            # matrix, factors, panel backups and the fill's element-pair blocks (4 per pair)
            fixed = 0 if cached else 6 * self.n * self.n * esz + 2 * self.n * 64 * esz
            return fixed + 8 * self.n * r * 16 + (1 << 20)
        ne = len(self.geometry) - 1
        mm = (self.n_modes or 40) + 2
        return ne * ne * mm * 20 * 16 + 4 * (2 * ne + 2) ** 2 * 16 + 8 * (2 * ne + 2) * 2 * r * 16 + (1 << 20)


class FactorCache:
    """LRU cache of resident 2-D system matrices and factors, bounded in bytes.

    An entry can be pinned by the requests that will read it (``pin`` / ``unpin``): pinned
    entries are never evicted, so a request admitted as a cache hit finds its factors when
    it runs.  ``used`` counts every resident entry's bytes; the engine's admission counts
    them against its memory budget next to the running requests."""

    def __init__(self, capacity_bytes):
        self.capacity = int(capacity_bytes)
        self.used = 0
        self.items = collections.OrderedDict()
        self.pins = collections.Counter()
        self.lock = threading.Lock()
        self.hits = 0
        self.misses = 0

    def contains(self, key):
        with self.lock:
            return key in self.items

    def get(self, key):
        with self.lock:
            e = self.items.get(key)
            if e is None:
                self.misses += 1
                return None
            self.items.move_to_end(key)
            self.hits += 1
            return e

    def pin(self, key):
        """Pin a resident entry; returns False (nothing pinned) when it is not resident."""
        with self.lock:
            if key not in self.items:
                return False
            self.pins[key] += 1
            return True

    def unpin(self, key):
        with self.lock:
            self.pins[key] -= 1
            if self.pins[key] <= 0:
                del self.pins[key]

    def _evict_to(self, limit):
        # least recently used unpinned entries first, until used <= limit (lock held); nothing
        # is evicted when the pinned entries alone exceed the limit
        pinned = sum(e['bytes'] for k, e in self.items.items() if self.pins.get(k, 0) > 0)
        if pinned > limit:
            return False
        for k in [k for k in self.items if self.pins.get(k, 0) == 0]:
            if self.used <= limit:
                break
            old = self.items.pop(k)
            self.used -= old['bytes']
        return self.used <= limit

    def shrink_to(self, limit):
        """Evict unpinned entries until at most ``limit`` bytes stay resident; True if reached."""
        with self.lock:
            return self._evict_to(max(0, int(limit)))

    def put(self, key, entry, nbytes):
        with self.lock:
            if nbytes > self.capacity or key in self.items:
                return
            if not self._evict_to(self.capacity - nbytes):
                return  # the rest is pinned: do not exceed the capacity
            entry['bytes'] = nbytes
            self.items[key] = entry
            self.used += nbytes


def admission_fits(in_use, est, cache_used, budget, running):
    """The engine's admission rule: a request fits when the running requests' estimates, its
    own and the resident factor cache stay within the budget, or when nothing else runs."""
    return in_use + est + cache_used <= budget or running == 0


class _Slot:
    def __init__(self, device):
        self.ctx = Context(device)
        self.stream = torch.cuda.Stream(device)


class ServingEngine:
    def __init__(self, slots=4, hbm_budget_bytes=None, cache_bytes=None, device=0, tol=None):
        require_cuda()
        self.device = int(device)
        torch.cuda.set_device(self.device)
        free, _total = torch.cuda.mem_get_info(self.device)
        self.budget = int(hbm_budget_bytes or 0.8 * free)
        self.cache = FactorCache(cache_bytes if cache_bytes is not None else self.budget // 4)
        self.tol = ops.MIXED_RCS_TOL if tol is None else float(tol)
        self.slots = [_Slot(self.device) for _ in range(int(slots))]
        self.pending = collections.deque()
        self.cv = threading.Condition()
        self.in_use = 0
        self.running = 0
        self.max_running = 0
        self.closed = False
        self.done = []
        self.t0 = None
        self.threads = [threading.Thread(target=self._worker, args=(s,), daemon=True) for s in self.slots]
        for t in self.threads:
            t.start()

    # ------------------------------------------------------------------ API
    def submit(self, req):
        fut = cf.Future()
        req.arrival = time.perf_counter()
        with self.cv:
            if self.closed:
                raise RuntimeError('engine is closed')
            if self.t0 is None:
                self.t0 = req.arrival
            est = req.estimate_bytes(cached=self.cache.contains(req.cache_key()))
            if est > self.budget:
                fut.set_exception(MemoryError(f'request {req.id} needs ~{est / 2**30:.2f} GiB, above the '
                                              f'{self.budget / 2**30:.2f} GiB device budget'))
                return fut
            self.pending.append((req, fut, est))
            self.cv.notify_all()
        return fut

    def close(self):
        """Stop the slot threads, drop the factor cache and return the slots' device
        workspaces (the engine's memory goes back to the caller)."""
        with self.cv:
            self.closed = True
            self.cv.notify_all()
        for t in self.threads:
            t.join()
        with self.cache.lock:
            self.cache.items.clear()
            self.cache.used = 0
        for slot in self.slots:
            slot.stream.synchronize()
            slot.ctx.lib.grim_release_workspace(slot.ctx.h)

    def stats(self):
        with self.cv:
            lat = np.array([r.finished - r.arrival for r in self.done])
            span = (max(r.finished for r in self.done) - self.t0) if self.done else 0.0
        out = {'completed': int(len(lat)), 'max_concurrent': int(self.max_running),
               'cache_hits': self.cache.hits, 'cache_misses': self.cache.misses}
        if len(lat):
            out.update(p50_ms=float(np.percentile(lat, 50) * 1e3), p99_ms=float(np.percentile(lat, 99) * 1e3),
                       mean_ms=float(lat.mean() * 1e3), solves_per_s=float(len(lat) / span) if span > 0 else None)
        return out

    # ------------------------------------------------------------------ scheduling
    def _take(self):
        """Admit the oldest pending request that fits next to the running ones and the
        resident factor cache (unpinned cache entries are evicted to make room).  A request
        whose factors are resident is estimated without them and pins them until it ends."""
        for i, (req, fut, _est) in enumerate(self.pending):
            key = req.cache_key()
            cached = self.cache.pin(key)
            est = req.estimate_bytes(cached=cached)
            if not admission_fits(self.in_use, est, self.cache.used, self.budget, self.running):
                self.cache.shrink_to(self.budget - self.in_use - est)
            if admission_fits(self.in_use, est, self.cache.used, self.budget, self.running):
                del self.pending[i]
                req.pinned = key if cached else None
                return req, fut, est
            if cached:
                self.cache.unpin(key)
        return None

    def _worker(self, slot):
        torch.cuda.set_device(self.device)
        while True:
            with self.cv:
                item = None
                while item is None:
                    if self.closed and not self.pending:
                        return
                    item = self._take()
                    if item is None:
                        self.cv.wait(timeout=0.05)
                req, fut, est = item
                self.in_use += est
                self.running += 1
                self.max_running = max(self.max_running, self.running)
            try:
                req.started = time.perf_counter()
                result = self._run(slot, req)
                req.finished = time.perf_counter()
                fut.set_result(result)
            except BaseException as exc:  # surfaced to the caller through the future
                req.finished = time.perf_counter()
                fut.set_exception(exc)
            finally:
                if getattr(req, 'pinned', None) is not None:
                    self.cache.unpin(req.pinned)
                    req.pinned = None
                with self.cv:
                    self.in_use -= est
                    self.running -= 1
                    if fut.exception() is None:
                        self.done.append(req)
                    self.cv.notify_all()

    # ------------------------------------------------------------------ execution
    def _run(self, slot, req):
        with torch.cuda.stream(slot.stream):
            slot.ctx.bind_stream(slot.stream)
            if req.kind == '2d':
                amp, tele = self._run_2d(slot, req)
                return {'id': req.id, 'amplitude': amp, 'telemetry': tele}
            from ..bor.solver import solve_bor_device, mode_limits
            mcap, _ = mode_limits(req.k, float(np.max(req.geometry[:, 0])), req.angles, req.n_modes)
            closed = req.geometry[0, 0] == 0.0 and req.geometry[-1, 0] == 0.0
            # the reference's default formulation: the CFIE for a closed body, else the EFIE
            F, tele = solve_bor_device(req.geometry, req.k, req.angles, mcap, precision=req.precision,
                                       tol=self.tol, ctx=slot.ctx, alpha=0.5 if closed else 1.0)
            nth = len(req.angles)
            return {'id': req.id, 'amp_vv': F[:nth], 'amp_hh': F[nth:], 'telemetry': tele}

    def _run_2d(self, slot, req):
        """A 2-D request in the reference's linear-Galerkin combined formulation: fill and a
        partial-pivoting factorization (kept in the cache), then the angles' solves guarded by
        the backward error (refinement for mixed precision, the FP64 gate for FP64)."""
        ctx, s = slot.ctx, slot.stream
        ang = torch.as_tensor(req.angles, device='cuda')
        key = req.cache_key()
        entry = self.cache.get(key)
        req.cache_hit = entry is not None
        mixed = req.precision == 'mixed'
        if entry is None:
            body = galerkin.GalerkinBody([req.geometry], ctx=ctx)
            n = body.n
            z = ops.fill(body, req.k, req.pol, complex64=mixed, ctx=ctx)
            lu = z.clone()
            ipiv = torch.empty(n, dtype=torch.int32, device='cuda')
            info = ctypes.c_int(0)
            fn = ctx.lib.grim_cgetrf if mixed else ctx.lib.grim_zgetrf
            _lib.check(ctx.lib.grim_set_tuning(ctx.h, _lib.TUNE_PIVOT, ops.PIVOTS[body.pivot]), 'grim_set_tuning')
            try:
                _lib.check(fn(ctx.h, n, ptr(lu), n, ptr(ipiv), ctypes.byref(info)), 'getrf')
            finally:
                ctx.lib.grim_set_tuning(ctx.h, _lib.TUNE_PIVOT, _lib.PIVOT_CERTIFIED)
            if info.value:
                raise _lib.GrimError(_lib.GRIM_ERR_SINGULAR, f'request {req.id}: singular system (info={info.value})')
            entry = {'z': z, 'lu': lu, 'ipiv': ipiv, 'body': body}
            self.cache.put(key, entry, 2 * z.numel() * z.element_size())
        else:
            body = entry['body']
            n = body.n
            for t in (entry['z'], entry['lu'], entry['ipiv']):
                t.record_stream(s)
        b = ops.rhs(body, req.k, req.pol, ang, ctx=ctx)
        tele = {'cache_hit': req.cache_hit, 'n': n}
        st = _lib.GrimSolveInfo()
        if mixed:
            b0 = b.clone()
            # the cached factor pivots partially: its solves keep the substitution kernels
            ctx.lib.grim_set_tuning(ctx.h, _lib.TUNE_PIVOT, _lib.PIVOT_PARTIAL)
            status = ctx.lib.grim_zgesv_mixed_factored(ctx.h, n, int(b.shape[0]), None, 0, ptr(entry['z']), n,
                                                       ptr(entry['lu']), ptr(entry['ipiv']), ptr(b), n, self.tol, 10,
                                                       ctypes.byref(st))
            ctx.lib.grim_set_tuning(ctx.h, _lib.TUNE_PIVOT, _lib.PIVOT_CERTIFIED)
            if status == _lib.GRIM_ERR_NOT_CONVERGED:
                # stalled refinement: solve this request in FP64 (reference mixed -> double ladder)
                z64 = ops.fill(body, req.k, req.pol, ctx=ctx)
                x = b0
                ops.solve_guarded(z64, x, pivot=body.pivot, ctx=ctx)
                tele['fp64_fallback'] = True
            else:
                _lib.check(status, 'grim_zgesv_mixed_factored')
                x = b
            tele.update(st.as_dict())
        else:
            x = b.clone()
            _lib.check(ctx.lib.grim_zgetrs(ctx.h, n, int(b.shape[0]), ptr(entry['lu']), n, ptr(entry['ipiv']), ptr(x),
                                           n), 'grim_zgetrs')
            berr = ops.backward_error(entry['z'], x, b, ctx=ctx)
            tele['backward_error'] = float(berr.max().item())
            if not tele['backward_error'] <= ops.DOUBLE_GATE_TOL:
                # the cached factor misses the FP64 gate: the gated solve of this request
                x = b.clone()
                st_g, berr = ops.solve_guarded(entry['z'], x, pivot=body.pivot, ctx=ctx)
                tele['backward_error'] = float(berr.max().item())
                tele['gate_fallback'] = st_g['gate_fallback']
        amp = ops.farfield(body, req.k, ang, x, ctx=ctx)
        return amp.cpu().numpy(), tele


def synthetic_stream(seed, count, nmax=8192, angle_max=720, repeat_fraction=0.3, bor_fraction=0.2,
                     bor_elements=120, precision='mixed'):
    """Seeded mixed request list (2-D superellipses/airfoils and BoR ogives)."""
    from .. import synthetic as S
    rng = np.random.default_rng(seed)
    reqs = []
    made = []
    for _ in range(count):
        nang = int(rng.integers(1, angle_max + 1))
        ang = np.sort(rng.uniform(0.0, 360.0, nang))
        if made and rng.random() < repeat_fraction:
            geom, k, pol = made[int(rng.integers(0, len(made)))]
            reqs.append(Request('2d', geom, k, ang, pol, precision))
            continue
        if rng.random() < bor_fraction:
            gen, length, half = S.ogive_case(int(rng.integers(0, 1 << 30)), n=bor_elements)
            k = float(rng.uniform(2.0, 12.0))
            mm = int(rng.integers(8, 41))
            th = np.sort(rng.uniform(0.0, 180.0, min(nang, 181)))
            reqs.append(Request('bor', gen, k, th, precision=precision, n_modes=mm))
            continue
        n = int(rng.integers(32, nmax // 2 + 1)) * 2
        if rng.random() < 0.5:
            v = S.superellipse(float(rng.uniform(0.3, 1.0)), float(rng.uniform(0.2, 0.8)), float(rng.uniform(1.5, 4.0)), n)
        else:
            v = S.naca_symmetric(float(rng.uniform(0.08, 0.15)), n)
        lam = S.polygon_perimeter(v) * 10.0 / n
        k = 2 * np.pi / lam
        pol = 'TM' if rng.random() < 0.5 else 'TE'
        made.append((v, k, pol))
        reqs.append(Request('2d', v, k, ang, pol, precision))
    gaps = rng.exponential(1.0, count)
    return reqs, gaps
