"""Execution scopes and environment settings of the GPU solve path.

Mirrors the reference's scoped options:
* ``linear_precision('double'|'mixed')`` -- ``linalg/refined_lu.py:13-22``;
* ``GHOST_DENSE_BACKEND`` in {cpu, auto, gpu} and ``GHOST_DENSE_GPU_MIN_N`` --
  ``twod/solver.py:291-311``, ``twod/constants.py:25-28``.  This package is the GPU
  backend and has no CPU solver, so ``cpu`` (a request for the reference's CPU LAPACK
  path) is refused with ``RuntimeError`` by every solve instead of running on the GPU
  unasked; ``auto`` and ``gpu`` both run on the GPU.

One scope has no counterpart in the reference, whose frequency workers are processes of
one host: ``shard_over_ranks(group)`` makes the public solves of every rank of a
``torch.distributed`` process group (one process per GPU) split the independent systems
of each request -- frequencies and polarisations of a 2-D request, Fourier modes of a
body of revolution -- between the ranks and gather the host results, so each rank
returns the whole result.
"""
from __future__ import annotations

import contextvars
import os
from contextlib import contextmanager

DENSE_GPU_BACKEND_ENV = 'GHOST_DENSE_BACKEND'
DENSE_GPU_MIN_N_ENV = 'GHOST_DENSE_GPU_MIN_N'
DENSE_GPU_MIN_N_DEFAULT = 768

_PRECISION = contextvars.ContextVar('grim_lu_precision', default='double')
_SHARD = contextvars.ContextVar('grim_shard_group', default=None)


@contextmanager
def linear_precision(value):
    if value not in {'double', 'mixed'}:
        raise ValueError('LU precision must be double or mixed.')
    token = _PRECISION.set(value)
    try:
        yield
    finally:
        _PRECISION.reset(token)


def requested_precision():
    return _PRECISION.get()


class _WholeWorld:
    """Marker: shard over the default process group."""


@contextmanager
def shard_over_ranks(group=None):
    """Split the systems of every public solve inside the scope over the ranks of
    ``group`` (the default process group when None).  Every rank of the group must make
    the same calls with the same arguments inside the scope (the gathers are collective)."""
    token = _SHARD.set(_WholeWorld if group is None else group)
    try:
        yield
    finally:
        _SHARD.reset(token)


def requested_shard_group():
    """(active, group) of the innermost ``shard_over_ranks`` scope; group None means the
    default process group."""
    g = _SHARD.get()
    if g is None:
        return False, None
    return True, (None if g is _WholeWorld else g)


def requested_dense_backend():
    backend = os.environ.get(DENSE_GPU_BACKEND_ENV, 'gpu').strip().lower()
    if backend not in {'cpu', 'auto', 'gpu'}:
        raise ValueError(f'{DENSE_GPU_BACKEND_ENV} must be cpu, auto, or gpu.')
    try:
        minimum_n = int(os.environ.get(DENSE_GPU_MIN_N_ENV, str(DENSE_GPU_MIN_N_DEFAULT)))
    except (TypeError, ValueError):
        raise ValueError(f'{DENSE_GPU_MIN_N_ENV} must be a positive integer.') from None
    if minimum_n < 1:
        raise ValueError(f'{DENSE_GPU_MIN_N_ENV} must be a positive integer.')
    return backend, minimum_n


def require_gpu_dense_backend():
    """Refuse ``GHOST_DENSE_BACKEND=cpu``: this package has no CPU solver to honour it."""
    backend, _ = requested_dense_backend()
    if backend == 'cpu':
        raise RuntimeError(f'{DENSE_GPU_BACKEND_ENV}=cpu selects the reference CPU solver, which this GPU package '
                           'does not provide; unset it or use auto/gpu.')
    return backend
