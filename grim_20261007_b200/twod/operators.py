"""Device pipeline of one 2-D monostatic solve: fill -> excitation -> LU solve -> far field.

Everything here runs in libgrimgpu kernels on the current torch stream; tensors are
torch CUDA tensors used only as device memory.  Column-major matrices are held in
tensors of shape (ncols, ld).  A body is either a pulse-basis ``DeviceBody`` (point-matched
EFIE / MFIE) or a linear-Galerkin ``galerkin.GalerkinBody`` (the reference's combined
formulation); ``fill``, ``rhs`` and ``farfield`` dispatch on it, the solve is the same.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from .. import _lib
from ..device import context, ptr

POL_CODE = {'TM': _lib.POL_TM, 'TE': _lib.POL_TE}

# Normwise backward-error target of the mixed path for RCS solves (a backward error of
# 1e-10 moves the currents by about cond x 1e-10, far below 0.05 dB); the linear-algebra
# hook keeps the reference RefinedLU's relative-residual test at 2e-12.
MIXED_RCS_TOL = 1e-10
MIXED_DROPIN_TOL = 2e-12
DOUBLE_GATE_TOL = 1e-12   # the reference's FP64 normwise backward-error gate (twod/solver.py:694-760)


def canonical_pol(pol):
    p = str(pol).strip().upper()
    if p in ('TM', 'HH', 'H', 'HORIZONTAL'):
        return 'TM'
    if p in ('TE', 'VV', 'V', 'VERTICAL'):
        return 'TE'
    raise ValueError(f'Unknown polarization {pol!r}.')


class DeviceBody:
    """Panel geometry resident in HBM: (n, 7) float64 and the TE diagonal correction."""

    def __init__(self, geom, te_diag=None, device=None):
        g = np.ascontiguousarray(np.asarray(geom, dtype=np.float64))
        if g.ndim != 2 or g.shape[1] != 7:
            raise ValueError('panel geometry must have shape (n, 7)')
        self.n = int(g.shape[0])
        self.geom = torch.from_numpy(g).to(device or 'cuda', non_blocking=True)
        self.te_diag = None
        if te_diag is not None:
            self.te_diag = torch.from_numpy(np.ascontiguousarray(te_diag, dtype=np.float64)).to(device or 'cuda')
        self.h2d_bytes = g.nbytes + (0 if te_diag is None else np.asarray(te_diag).nbytes)


def fill(body, k, pol, complex64=False, out=None, ctx=None):
    if hasattr(body, 'fill_matrix'):  # linear-Galerkin body (galerkin.GalerkinBody)
        return body.fill_matrix(k, canonical_pol(pol), complex64=complex64, out=out, ctx=ctx)
    ctx = ctx or context()
    n = body.n
    dt = torch.complex64 if complex64 else torch.complex128
    z = out if out is not None else torch.empty((n, n), dtype=dt, device=body.geom.device)
    diag = body.te_diag if (canonical_pol(pol) == 'TE' and body.te_diag is not None) else None
    _lib.check(ctx.lib.grim_fill2d(ctx.h, POL_CODE[canonical_pol(pol)], n, ptr(body.geom), ptr(diag), float(k),
                                   ptr(z), n, int(complex64)), 'grim_fill2d')
    return z


def rhs(body, k, pol, angles_dev, complex64=False, out=None, ctx=None):
    if hasattr(body, 'rhs_matrix'):
        return body.rhs_matrix(k, canonical_pol(pol), angles_dev, complex64=complex64, out=out, ctx=ctx)
    ctx = ctx or context()
    n, nang = body.n, int(angles_dev.numel())
    dt = torch.complex64 if complex64 else torch.complex128
    b = out if out is not None else torch.empty((nang, n), dtype=dt, device=body.geom.device)
    _lib.check(ctx.lib.grim_rhs2d(ctx.h, POL_CODE[canonical_pol(pol)], n, ptr(body.geom), nang, ptr(angles_dev),
                                  float(k), ptr(b), n, int(complex64)), 'grim_rhs2d')
    return b


def farfield(body, k, angles_dev, x, out=None, ctx=None):
    if hasattr(body, 'far_amplitude'):
        return body.far_amplitude(k, angles_dev, x, out=out, ctx=ctx)
    ctx = ctx or context()
    nang = int(angles_dev.numel())
    amp = out if out is not None else torch.empty(nang, dtype=torch.complex128, device=body.geom.device)
    _lib.check(ctx.lib.grim_farfield2d(ctx.h, body.n, ptr(body.geom), nang, ptr(angles_dev), float(k), ptr(x),
                                       body.n, int(x.dtype == torch.complex64), ptr(amp)), 'grim_farfield2d')
    return amp


PIVOTS = {'certified': _lib.PIVOT_CERTIFIED, 'static': _lib.PIVOT_STATIC, 'partial': _lib.PIVOT_PARTIAL,
          'tournament': _lib.PIVOT_TOURNAMENT}


def solve_guarded(z, b, pivot='partial', tol=DOUBLE_GATE_TOL, max_refine=2, ctx=None):
    """FP64 solve of Z X = B with the reference's dense gate (``grim_zgesv_guarded``): LU in
    the ``pivot`` mode ('partial', 'tournament', 'certified' or 'static'), the per-column normwise
    backward error, at most ``max_refine`` refinement steps while it exceeds ``tol`` and a
    certified factorization when the gate still fails.  X overwrites ``b``; returns
    (telemetry dict, per-column backward errors on the device)."""
    ctx = ctx or context()
    n, nrhs = int(b.shape[1]), int(b.shape[0])
    berr = torch.empty(nrhs, dtype=torch.float64, device=b.device)
    info = ctypes.c_int(0)
    st = _lib.GrimSolveInfo()
    _lib.check(ctx.lib.grim_zgesv_guarded(ctx.h, n, nrhs, ptr(z), n, ptr(b), n, PIVOTS[pivot], float(tol),
                                          int(max_refine), ptr(berr), ctypes.byref(info), ctypes.byref(st)),
               'grim_zgesv_guarded')
    tele = st.as_dict()
    tele['pivot'] = pivot
    tele['gate_fallback'] = tele['pivoted_panels'] < 0
    return tele, berr


def solve_inplace(z, b, precision='double', tol=None, max_iter=10, z32=None, ctx=None, stop='relres', tuned=True,
                  pivot='certified'):
    """Solve Z X = B on the device; X overwrites ``b`` (complex128, shape (nrhs, n)).

    precision 'double': FP64 LU + triangular solves.  'mixed': complex64 LU of ``z32``
    (or of ``z`` rounded) with FP64 residual and update against ``z`` (complex128) or,
    when ``z`` is None, against the exact promotion of ``z32``; the refinement stops when
    every column's relative residual (``stop='relres'``, the reference RefinedLU test) or
    normwise backward error (``stop='berr'``) is <= ``tol``.  With ``tuned`` the handle's
    tile shapes come from the autotuner's cache (``tuning.apply``).
    ``pivot``: the factorization's pivot mode -- 'certified' (diagonal pivots, certified per
    panel, partial pivoting where they fail), 'partial' (partial pivoting throughout),
    'tournament' (tournament pivoting throughout) or
    'static' (diagonal pivots; the refinement guards the solution, a stall raises
    ``GrimNotConverged``).
    Returns the solve telemetry dict.
    """
    ctx = ctx or context()
    n = int(b.shape[1])
    nrhs = int(b.shape[0])
    info = ctypes.c_int(0)
    st = _lib.GrimSolveInfo()
    if precision == 'mixed':
        mode = _lib.PREC_MIXED_BERR if stop == 'berr' else _lib.PREC_MIXED
        if tuned:
            from .. import tuning
            tuning.apply(ctx, n, nrhs)
    else:
        mode = _lib.PREC_FP64
    if pivot == 'partial':
        mode |= _lib.PREC_PARTIAL_PIVOT
    elif pivot == 'tournament':
        mode |= _lib.PREC_TOURNAMENT_PIVOT
    elif pivot == 'static':
        mode |= _lib.PREC_STATIC_PIVOT
    tol = MIXED_DROPIN_TOL if tol is None else float(tol)
    status = ctx.lib.grim_zgesv_mixed(ctx.h, n, nrhs, ptr(z), n, ptr(z32), n, ptr(b), n, mode, tol, int(max_iter),
                                      ctypes.byref(info), ctypes.byref(st))
    _lib.check(status, 'grim_zgesv_mixed')
    return st.as_dict()


def condition_estimate(z, ctx=None):
    """cond_1 of the row/column-equilibrated ``z`` (complex128 device matrix), the reference's
    ``condition_est`` (twod/solver.py:529 ``_equilibrated_condition_from_lu``): ||B||_1 times
    the Hager-Higham estimate of ||B^-1||_1 on the device (``grim_zcond1_equilibrated``);
    ``inf`` for an exactly singular matrix."""
    ctx = ctx or context()
    if z.dtype != torch.complex128:
        raise TypeError('condition_estimate needs the complex128 matrix')
    out = ctypes.c_double(0.0)
    n = int(z.shape[0])
    _lib.check(ctx.lib.grim_zcond1_equilibrated(ctx.h, n, ptr(z), n, ctypes.byref(out)), 'grim_zcond1_equilibrated')
    return float(out.value)


def backward_error(z, x, b, ctx=None):
    """Per-column normwise backward error on the device (reference twod/solver.py:695-720)."""
    ctx = ctx or context()
    n, nrhs = int(b.shape[1]), int(b.shape[0])
    berr = torch.empty(nrhs, dtype=torch.float64, device=b.device)
    _lib.check(ctx.lib.grim_backward_error(ctx.h, n, nrhs, ptr(z), n, int(z.dtype == torch.complex64), ptr(x), n,
                                           ptr(b), n, ptr(berr)), 'grim_backward_error')
    return berr


def monostatic_solve(body, k, angles_deg, pol, precision='double', tol=None, check_backward_error=True,
                     angles_dev=None, keep=False, ctx=None, condition=False):
    """One (geometry, frequency, polarization) solve with all its angles, on the device.

    Returns dict(amplitude=<device complex128 (nang,)>, telemetry).  With precision
    'double' the system is filled in FP64, factored and solved in FP64 and its normwise
    backward error computed (the reference's 1e-12 gate); with 'mixed' a pulse-basis
    system is filled in complex64 (FP64 small-kR and self terms), factored in complex64
    and refined with FP64 residuals against that matrix, a linear-Galerkin system is
    filled in FP64, its complex64 rounding factored and the refinement run against the
    FP64 matrix.
    """
    pol = canonical_pol(pol)
    dev = body.geom.device
    if angles_dev is None:
        angles_dev = torch.as_tensor(np.asarray(angles_deg, dtype=np.float64), device=dev)
    # linear-Galerkin systems: partial pivoting leaves the diagonal, so they factor with
    # partial pivoting throughout and the FP64 path applies the reference's gate
    pivot = getattr(body, 'pivot', 'certified')
    static = pivot != 'certified'
    tele = {}
    if precision == 'mixed':
        b = rhs(body, k, pol, angles_dev, ctx=ctx)
        b0 = b.clone()
        if static:
            # linear-Galerkin systems fill in FP64 arithmetic whatever the output type, so
            # the refinement runs against the FP64 matrix (its complex64 rounding is
            # factored): the solution converges to the FP64 system's, not to the rounded one's
            z = fill(body, k, pol, ctx=ctx)
            z32 = None
        else:
            z = None
            z32 = fill(body, k, pol, complex64=True, ctx=ctx)
        try:
            st = solve_inplace(z, b, 'mixed', tol=MIXED_RCS_TOL if tol is None else tol, z32=z32, ctx=ctx,
                               stop='berr', pivot=pivot)
            x = b
            if z is None:
                z = z32
        except _lib.GrimNotConverged:
            # refinement stalled (ill-conditioned system): fall back to the FP64 path, as the
            # reference's mixed -> double ladder does (linalg/dense.py:74-98)
            if z is None or z.dtype != torch.complex128:
                z = fill(body, k, pol, ctx=ctx)
            x = b0
            if static:
                st, _berr = solve_guarded(z, x, pivot=pivot, ctx=ctx)
            else:
                st = solve_inplace(z, x, 'double', ctx=ctx)
            st['fp64_fallback'] = True
        tele.update(st)
    elif static:
        z = fill(body, k, pol, ctx=ctx)
        x = rhs(body, k, pol, angles_dev, ctx=ctx)
        st, berr = solve_guarded(z, x, pivot=pivot, ctx=ctx)
        tele.update(st)
        tele['backward_error_dev'] = berr
    else:
        z = fill(body, k, pol, ctx=ctx)
        b = rhs(body, k, pol, angles_dev, ctx=ctx)
        x = b.clone() if check_backward_error else b
        st = solve_inplace(z, x, 'double', ctx=ctx)
        tele.update(st)
        if check_backward_error:
            berr = backward_error(z, x, b, ctx=ctx)
            tele['backward_error_dev'] = berr
    if condition:
        # the estimate is of the FP64 system (filled again when the solve kept only complex64)
        z64 = z if z.dtype == torch.complex128 else fill(body, k, pol, ctx=ctx)
        tele['condition_est'] = condition_estimate(z64, ctx=ctx)
    amp = farfield(body, k, angles_dev, x, ctx=ctx)
    out = dict(amplitude=amp, telemetry=tele)
    if keep:
        out.update(matrix=z, solution=x)
    return out


def monostatic_solves_grouped(bodies, ks, angles_deg, pol, precision='mixed', tol=None, angles_dev=None,
                              use_graph=True, workers=4, condition=False):
    """Many (geometry, frequency, polarization) systems with one angle set -- the systems
    of a frequency sweep; ``pol`` is one polarization or one per system -- solved
    together: fills and excitations on the device
    worker pool, ONE grouped LU of all matrices (``grouped.getrf_grouped``, a captured CUDA
    graph), then per system the triangular solves, the FP64 refinement (mixed) or backward
    error (double) and the far field on the pool.  Same numerics per system as
    ``monostatic_solve`` (the grouped factors equal the single-system ones), including the
    mixed -> double fallback of a stalled refinement.  Returns [dict(amplitude, telemetry)]
    in input order.
    """
    from ..device import run_pool
    from ..grouped import getrf_grouped, refine_factored
    from .. import tuning
    if not bodies:
        return []
    pols = [canonical_pol(pol)] * len(bodies) if isinstance(pol, str) else [canonical_pol(p) for p in pol]
    dev = bodies[0].geom.device
    if angles_dev is None:
        angles_dev = torch.as_tensor(np.asarray(angles_deg, dtype=np.float64), device=dev)
    nang = int(angles_dev.numel())
    mixed = precision == 'mixed'
    tol = MIXED_RCS_TOL if tol is None else float(tol)
    costs = [float(b.n) ** 3 + nang * float(b.n) ** 2 for b in bodies]

    def prep(i):
        def run():
            c = context()
            z = fill(bodies[i], ks[i], pols[i], complex64=mixed, ctx=c)
            b = rhs(bodies[i], ks[i], pols[i], angles_dev, ctx=c)
            return {'z': z, 'lu': z.clone(), 'b': b}
        return run

    if any(getattr(b, 'pivot', 'certified') in ('partial', 'tournament') for b in bodies):
        # the grouped factorization keeps diagonal pivots; systems that need partial
        # pivoting are factored one by one on the pool instead
        jobs = [(lambda i=i: monostatic_solve(bodies[i], ks[i], angles_deg, pols[i], precision=precision, tol=tol,
                                              angles_dev=angles_dev, condition=condition))
                for i in range(len(bodies))]
        return run_pool(jobs, workers=workers, costs=costs)
    static = all(getattr(b, 'pivot', 'certified') == 'static' for b in bodies)
    parts = run_pool([prep(i) for i in range(len(bodies))], workers=workers, costs=costs)
    ipivs, infos, piv = getrf_grouped([p['lu'] for p in parts], use_graph=use_graph, static_pivot=static)
    for i, inf in enumerate(infos):
        if inf and not static:
            raise _lib.GrimError(_lib.GRIM_ERR_SINGULAR, f'system {i} (n={bodies[i].n}) is exactly singular '
                                                         f'(info={inf})')

    def finish(i):
        def run():
            c = context()
            p = parts[i]
            tele = {'grouped': True, 'pivoted_panels': piv[i]}
            if mixed:
                tuning.apply(c, bodies[i].n, nang)
                b0 = p['b'].clone()
                try:
                    st = refine_factored(p['z'], p['lu'], ipivs[i], p['b'], tol, stop='berr', ctx=c)
                    x = p['b']
                except _lib.GrimNotConverged:
                    z64 = fill(bodies[i], ks[i], pols[i], ctx=c)
                    x = b0
                    if static:
                        st, _berr = solve_guarded(z64, x, pivot='static', ctx=c)
                    else:
                        st = solve_inplace(z64, x, 'double', ctx=c)
                    st['fp64_fallback'] = True
            else:
                x = p['b'].clone()
                n = bodies[i].n
                _lib.check(c.lib.grim_zgetrs(c.h, n, nang, ptr(p['lu']), n, ptr(ipivs[i]), ptr(x), n), 'grim_zgetrs')
                berr = backward_error(p['z'], x, p['b'], ctx=c)
                st = {'precision_mode': _lib.PREC_FP64, 'backward_error_dev': berr}
                if static and (infos[i] or not float(berr.max()) <= DOUBLE_GATE_TOL):
                    # the static-pivot factor missed the gate: the guarded solve of this system
                    x = p['b'].clone()
                    st, berr = solve_guarded(p['z'], x, pivot='static', ctx=c)
                    st['backward_error_dev'] = berr
            tele.update(st)
            if condition:
                z64 = p['z'] if p['z'].dtype == torch.complex128 else fill(bodies[i], ks[i], pols[i], ctx=c)
                tele['condition_est'] = condition_estimate(z64, ctx=c)
            amp = farfield(bodies[i], ks[i], angles_dev, x, ctx=c)
            # release this system's matrices as soon as its work is queued: they were
            # allocated on another worker's stream, so the allocator must wait for this one
            cur = torch.cuda.current_stream()
            for t in p.values():
                t.record_stream(cur)
            p.clear()
            return dict(amplitude=amp, telemetry=tele)
        return run

    return run_pool([finish(i) for i in range(len(bodies))], workers=workers, costs=costs)


def sigma_2d(amp, k):
    return 0.25 / float(k) * np.abs(amp) ** 2


def sigma_db(sigma, floor=1e-12):
    return 10.0 * np.log10(np.maximum(sigma, floor))
