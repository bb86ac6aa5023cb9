"""Grouped factorization of many independent systems of different orders.

The reference factors the systems of a frequency sweep one per worker process
(``execution/frequency_sweep.py:140-188``, ``_plan`` / ``_compute``) and the Fourier modes
of a body of revolution one after another (``bor/solver.py:2827-3250`` with
``bor/factor.py:120`` ``ModalFactor`` per mode).  Here all of them are factored by ONE
sequence of launches (``grim_getrf_grouped``): every 64-column step is one launch per stage
over all systems still active, so the latency-bound panel chain of one system (its
diagonal block and panel solve) runs beside the same stages of every other system, and the
trailing updates of all systems fill the GPU together.  The sequence is captured in a CUDA
graph on the handle and replayed while the orders stay the same.  The triangular solves
and FP64 refinement that follow run per system on the device worker pool.
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib
from .device import context, ptr, run_pool


def getrf_grouped(mats, use_graph=True, ctx=None, static_pivot=False):
    """Factor the square column-major device matrices ``mats`` in place (all complex64 or all
    complex128, contiguous, leading dimension = order) with one grouped LU.

    Returns (ipivs, infos, pivoted): 1-based int32 pivots per system, LAPACK-style info per
    system (0, or k+1 for an exactly zero U(k,k)) and the number of panels that fell back to
    partial pivoting.  The factors equal ``grim_cgetrf`` / ``grim_zgetrf`` of each matrix.
    With ``static_pivot`` every system keeps its diagonal pivots (no partial-pivoting
    fallback); the caller guards the solutions.
    """
    ctx = ctx or context()
    mats = list(mats)
    if not mats:
        return [], [], []
    dt = mats[0].dtype
    if dt not in (torch.complex64, torch.complex128):
        raise TypeError('getrf_grouped: complex64 or complex128 matrices')
    for m in mats:
        if m.dtype != dt or m.dim() != 2 or m.shape[0] != m.shape[1] or not m.is_contiguous() or not m.is_cuda:
            raise ValueError('getrf_grouped: square contiguous device matrices of one dtype')
    count = len(mats)
    ipivs = [torch.empty(int(m.shape[0]), dtype=torch.int32, device=m.device) for m in mats]
    ns = (ctypes.c_int * count)(*[int(m.shape[0]) for m in mats])
    lds = (ctypes.c_int64 * count)(*[int(m.shape[0]) for m in mats])
    aps = (ctypes.c_void_p * count)(*[m.data_ptr() for m in mats])
    pps = (ctypes.c_void_p * count)(*[p.data_ptr() for p in ipivs])
    info = (ctypes.c_int * count)()
    piv = (ctypes.c_int * count)()
    _lib.check(ctx.lib.grim_set_tuning(ctx.h, _lib.TUNE_PIVOT, _lib.PIVOT_STATIC if static_pivot else
                                       _lib.PIVOT_CERTIFIED), 'grim_set_tuning')
    try:
        _lib.check(ctx.lib.grim_getrf_grouped(ctx.h, count, ns, aps, lds, pps, int(dt == torch.complex64),
                                              int(use_graph), info, piv), 'grim_getrf_grouped')
    finally:
        ctx.lib.grim_set_tuning(ctx.h, _lib.TUNE_PIVOT, _lib.PIVOT_CERTIFIED)
    return ipivs, list(info), list(piv)


def refine_factored(z, lu32, ipiv, b, tol, stop='berr', max_iter=10, ctx=None):
    """FP64 refinement of the complex64 factorization ``lu32`` / ``ipiv`` of ``z`` (complex128,
    or complex64 whose exact promotion is the system) for the right-hand sides ``b``
    (complex128, (nrhs, n)); X overwrites ``b``.  Raises GrimNotConverged when the
    refinement stalls.  Returns the solve telemetry dict."""
    ctx = ctx or context()
    n, nrhs = int(b.shape[1]), int(b.shape[0])
    mode = _lib.PREC_MIXED_BERR if stop == 'berr' else _lib.PREC_MIXED
    st = _lib.GrimSolveInfo()
    z64, z32 = (z, None) if z.dtype == torch.complex128 else (None, z)
    status = ctx.lib.grim_zgesv_refine_factored(ctx.h, n, nrhs, ptr(z64), n, ptr(z32), n, ptr(lu32), ptr(ipiv), ptr(b),
                                                n, mode, float(tol), int(max_iter), ctypes.byref(st))
    _lib.check(status, 'grim_zgesv_refine_factored')
    return st.as_dict()


def solve_grouped(zs, bs, precision='mixed', tol=None, stop='berr', use_graph=True, workers=4, costs=None,
                  keep_factors=False):
    """Solve Z_i X_i = B_i for every system: one grouped LU of all matrices, then the
    triangular solves (and, mixed, the FP64 refinement) per system on the worker pool.

    ``zs``: column-major device matrices, kept (complex128, or for mixed complex64 whose exact
    promotion is the system); the LU runs in complex64 (mixed) or complex128 (double);
    ``bs``: complex128 (nrhs_i, n_i) right-hand sides, overwritten by the solutions.
    Returns per-system telemetry dicts; a mixed system whose refinement stalls carries
    ``not_converged=True`` and its ``bs`` entry is left as the partial solution.  With
    ``keep_factors`` every dict also holds its factor: ``lu`` (complex64 for mixed, else
    complex128, LAPACK layout) and ``ipiv`` (1-based int32), both on the device.
    """
    from .twod.operators import MIXED_RCS_TOL
    lus = [z.to(torch.complex64, copy=True) if precision == 'mixed' else z.clone() for z in zs]
    ipivs, infos, piv = getrf_grouped(lus, use_graph=use_graph)
    for i, inf in enumerate(infos):
        if inf:
            raise _lib.GrimError(_lib.GRIM_ERR_SINGULAR, f'grouped factorization: system {i} is exactly singular '
                                                         f'(info={inf})')
    tol = MIXED_RCS_TOL if tol is None else float(tol)

    def job(i):
        def run():
            c = context()
            if precision == 'mixed':
                try:
                    st = refine_factored(zs[i], lus[i], ipivs[i], bs[i], tol, stop=stop, ctx=c)
                except _lib.GrimNotConverged:
                    st = {'not_converged': True}
            else:
                n, nrhs = int(bs[i].shape[1]), int(bs[i].shape[0])
                _lib.check(c.lib.grim_zgetrs(c.h, n, nrhs, ptr(lus[i]), n, ptr(ipivs[i]), ptr(bs[i]), n), 'grim_zgetrs')
                st = {'precision_mode': _lib.PREC_FP64}
            st['pivoted_panels'] = piv[i]
            st['grouped'] = True
            if keep_factors:
                st['lu'], st['ipiv'] = lus[i], ipivs[i]
            return st
        return run

    return run_pool([job(i) for i in range(len(zs))], workers=workers, costs=costs)
