"""Device context: one libgrimgpu handle per CUDA device, bound to torch's current stream.

PyTorch provides device memory (its caching allocator), pinned host buffers and the
stream; all arithmetic runs in libgrimgpu's kernels.  Matrices live in torch tensors
of shape (ncols, ld): row c of the tensor is column c of the column-major matrix.
"""
from __future__ import annotations

import ctypes
import threading

import numpy as np
import torch

from . import _lib

_contexts = {}
_ctx_lock = threading.Lock()


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
    with _ctx_lock:
        ctx = _contexts.get(dev)
        if ctx is None:
            ctx = Context(dev)
            _contexts[dev] = ctx
    ctx.bind_stream()
    return ctx


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
