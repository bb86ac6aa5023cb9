"""Device context: one libgrimgpu handle per CUDA device, bound to torch's current stream.

PyTorch provides device memory (its caching allocator), pinned host buffers and the
stream; all arithmetic runs in libgrimgpu's kernels.  Matrices live in torch tensors
of shape (ncols, ld): row c of the tensor is column c of the column-major matrix.

Independent solves (the two co-polarised channels of a 2-D solve, the systems of a
sweep) overlap on the GPU through ``run_concurrent``: each runs in its own host thread
on a worker -- its own libgrimgpu handle (workspaces, error flag) and CUDA stream --
so one solve's latency-bound panel chain runs beside another's tensor-core updates.
"""
from __future__ import annotations

import contextlib
import contextvars
import ctypes
import queue
import threading
from concurrent.futures import Future

import numpy as np
import torch

from . import _lib

_contexts = {}
_ctx_lock = threading.Lock()
_workers = {}  # (device, index) -> (Context, torch.cuda.Stream)
_tls = threading.local()  # per-thread override of context() inside a worker


def require_cuda():
    if not torch.cuda.is_available():
        raise _lib.GrimError(_lib.GRIM_ERR_CUDA, 'no CUDA device is available; the GPU solve path has no CPU fallback')


class Context:
    def __init__(self, device=0):
        require_cuda()
        self.lib = _lib.load()
        self.device = int(device)
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.check(self.lib.grim_create(self.device, ctypes.byref(h)), 'grim_create')
        self.h = h
        buf = ctypes.create_string_buffer(256)
        _lib.check(self.lib.grim_device_name(self.h, buf, 256), 'grim_device_name')
        self.device_name = buf.value.decode(errors='replace')
        self._bound_stream = None

    def bind_stream(self, stream=None):
        """Run library kernels on ``stream`` (default: torch's current stream)."""
        s = torch.cuda.current_stream(self.device) if stream is None else stream
        ptr = s.cuda_stream
        if ptr != self._bound_stream:
            _lib.check(self.lib.grim_set_stream(self.h, ctypes.c_void_p(ptr)), 'grim_set_stream')
            self._bound_stream = ptr
        return s

    @property
    def launches(self):
        return int(self.lib.grim_launch_count(self.h))

    def mem_info(self):
        f, t = ctypes.c_size_t(), ctypes.c_size_t()
        _lib.check(self.lib.grim_mem_info(self.h, ctypes.byref(f), ctypes.byref(t)), 'grim_mem_info')
        return int(f.value), int(t.value)

    def release_workspace(self):
        _lib.check(self.lib.grim_release_workspace(self.h), 'grim_release_workspace')

    def close(self):
        if self.h:
            self.lib.grim_destroy(self.h)
            self.h = None


def context(device=None):
    require_cuda()
    dev = torch.cuda.current_device() if device is None else int(device)
    over = getattr(_tls, 'ctx', None)
    if over is not None and over.device == dev:
        over.bind_stream()
        return over
    with _ctx_lock:
        ctx = _contexts.get(dev)
        if ctx is None:
            ctx = Context(dev)
            _contexts[dev] = ctx
    ctx.bind_stream()
    return ctx


_busy = set()  # (device, index) of workers held by a running pool
_threads = {}  # (device, index) -> task queue of the worker's host thread


def _worker_queue(dev, index):
    """Task queue of worker ``index``'s host thread (started on first use and kept, so a
    pool call does not start and join threads).  A worker index is held by one pool at a
    time (``_acquire``), so its thread runs one pool's loop at a time."""
    with _ctx_lock:
        q = _threads.get((dev, index))
        if q is None:
            q = queue.SimpleQueue()

            def serve(q=q):
                while True:
                    fn, fut = q.get()
                    if not fut.set_running_or_notify_cancel():
                        continue
                    try:
                        fut.set_result(fn())
                    except BaseException as exc:  # noqa: BLE001 - delivered to the pool's caller
                        fut.set_exception(exc)

            threading.Thread(target=serve, daemon=True, name=f'grim-worker-{dev}-{index}').start()
            _threads[(dev, index)] = q
    return q


def _worker(dev, index):
    with _ctx_lock:
        w = _workers.get((dev, index))
        if w is None:
            with torch.cuda.device(dev):
                w = (Context(dev), torch.cuda.Stream(dev))
            _workers[(dev, index)] = w
    return w


def _acquire(dev, count):
    """Indices of ``count`` workers no other pool holds (new ones are created on demand), so
    that pools started from different host threads never share a handle or a stream."""
    with _ctx_lock:
        got, i = [], 0
        while len(got) < count:
            if (dev, i) not in _busy:
                _busy.add((dev, i))
                got.append(i)
            i += 1
    return got


def _release(dev, indices):
    with _ctx_lock:
        for i in indices:
            _busy.discard((dev, i))


def all_contexts(device=None):
    """The default context and every worker context created so far on ``device``."""
    dev = torch.cuda.current_device() if device is None else int(device)
    out = [context(dev)]
    with _ctx_lock:
        out += [w[0] for (d, _), w in sorted(_workers.items()) if d == dev]
    return out


@contextlib.contextmanager
def worker(index, device=None):
    """Route this thread's library calls (``context()``) and torch work to worker ``index``."""
    dev = torch.cuda.current_device() if device is None else int(device)
    ctx, stream = _worker(dev, index)
    prev = getattr(_tls, 'ctx', None)
    _tls.ctx = ctx
    try:
        with torch.cuda.device(dev), torch.cuda.stream(stream):
            ctx.bind_stream(stream)
            yield ctx, stream
    finally:
        _tls.ctx = prev


def _record_on(obj, stream):
    """Mark every CUDA tensor in a result (a tensor, or dicts and tuples nesting them) as used by
    ``stream`` (caching-allocator safety).  Lists are host data (sample records) and are not
    searched."""
    if isinstance(obj, torch.Tensor):
        if obj.is_cuda:
            obj.record_stream(stream)
    elif isinstance(obj, dict):
        for v in obj.values():
            if isinstance(v, (torch.Tensor, dict, tuple)):
                _record_on(v, stream)
    elif isinstance(obj, tuple):
        for v in obj:
            _record_on(v, stream)


def in_worker():
    """True inside a worker thread (nested pools run their tasks in place)."""
    return getattr(_tls, 'ctx', None) is not None


def run_pool(fns, workers=None, costs=None, on_done=None, device=None):
    """Run the callables ``fns`` on up to ``workers`` device workers and return their results
    in input order.

    Each worker is a host thread with its own libgrimgpu handle and CUDA stream; it takes
    the next task from a shared queue, largest ``costs`` first (longest-processing-time
    order), so independent solves of different sizes overlap on the GPU.  Worker streams
    first wait for the work already queued on the caller's current stream; the caller's
    stream then waits for every worker, so results (device tensors included) can be used
    on it directly.  Every task runs in a copy of the caller's context variables
    (``linear_precision`` and other scoped options apply inside it).  ``on_done(i, result)``
    is called (serialised) as each task finishes.  The first exception raised by a task is
    re-raised after the running tasks finish; tasks not yet started are skipped.  Called
    from inside a worker, the tasks run in place, one after another.
    """
    fns = list(fns)
    if not fns:
        return []
    if workers is None:
        workers = len(fns)
    workers = max(1, min(int(workers), len(fns)))
    if in_worker() or workers == 1:
        out = []
        for i, f in enumerate(fns):
            r = f()
            if on_done is not None:
                on_done(i, r)
            out.append(r)
        return out
    dev = torch.cuda.current_device() if device is None else int(device)
    caller = torch.cuda.current_stream(dev)
    ready = torch.cuda.Event()
    ready.record(caller)
    order = list(range(len(fns)))
    if costs is not None:
        order.sort(key=lambda i: -float(costs[i]))
    lock = threading.Lock()
    state = {'next': 0, 'error': None}
    results = [None] * len(fns)
    scopes = [contextvars.copy_context() for _ in fns]

    def take():
        with lock:
            if state['error'] is not None or state['next'] >= len(order):
                return None
            i = order[state['next']]
            state['next'] += 1
            return i

    held = _acquire(dev, workers)

    def loop(w):
        with worker(held[w], dev) as (_ctx, stream):
            stream.wait_event(ready)
            while True:
                i = take()
                if i is None:
                    break
                try:
                    r = scopes[i].run(fns[i])
                except BaseException as exc:  # noqa: BLE001 - re-raised in the caller
                    with lock:
                        if state['error'] is None:
                            state['error'] = exc
                    break
                results[i] = r
                if on_done is not None:
                    with lock:
                        on_done(i, r)
            done = torch.cuda.Event()
            done.record(stream)
            return done

    try:
        futs = []
        for w in range(workers):
            fut = Future()
            _worker_queue(dev, held[w]).put((lambda w=w: loop(w), fut))
            futs.append(fut)
        events = [fut.result() for fut in futs]
    finally:
        _release(dev, held)
    for done in events:
        caller.wait_event(done)
    if state['error'] is not None:
        raise state['error']
    for r in results:
        _record_on(r, caller)
    return results


def run_concurrent(fns, device=None):
    """Run the callables ``fns`` at once, fns[i] on its own worker (see ``run_pool``)."""
    fns = list(fns)
    return run_pool(fns, workers=len(fns), device=device)


def ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def to_device_colmajor(a, dtype=torch.complex128, device=None):
    """numpy (m, n) matrix -> device tensor (n, m) holding it column-major."""
    a = np.asarray(a)
    if a.ndim == 1:
        a = a[:, None]
    host = torch.from_numpy(np.ascontiguousarray(a.T).astype(np.complex128 if dtype == torch.complex128 else np.complex64,
                                                              copy=False))
    return host.to(device=device or 'cuda', dtype=dtype, non_blocking=False)


def to_host_matrix(t):
    """Device tensor (n, m) in column-major layout -> numpy (m, n) F-ordered matrix."""
    return t.detach().cpu().numpy().T
