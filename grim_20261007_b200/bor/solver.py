"""Body-of-revolution monostatic RCS on the GPU (reference ``bor/solver.py:4066`` ``solve_bor``).

Pipeline per frequency (all arithmetic in libgrimgpu kernels):
  1. ``grim_bor_moments``: mode-independent element-pair moments of the modal Green's
     function and, for the CFIE / MFIE, of the modal MFIE brackets, for n = 0..m_max+1
     (far pairs, near work items and their reduction: three launches);
  2. per signed mode m = -m_max..m_max: ``grim_bor_assemble`` (reduced matrix with the
     axis-pole treatment), ``grim_bor_excitation`` (VV/HH right-hand sides for every aspect
     and the far-field weights), dense solve (``grim_zgesv_mixed``, FP64 or mixed),
     ``grim_bor_farfield_accumulate``;
  3. sigma = 4 pi |F|^2 with F = -(j k eta / 4 pi) sum_m W_m^T x_m.

The PEC EFIE, MFIE and CFIE are implemented (the reference's default for a closed body is
the CFIE with alpha = 0.5).  Impedance and sheet models are rejected.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from .. import _lib
from .. import sharding
from ..device import context, ptr, require_cuda, run_pool
from ..execution import requested_precision, requested_shard_group
from ..twod import operators as ops2d
from .rules import near_rules, pair_classes

ETA0 = 376.730313668
C0 = 299_792_458.0
FAR_ORDER = 3
MAX_NXI = 8192


def validate_generatrix(points):
    p = np.asarray(points, dtype=np.float64)
    if p.ndim != 2 or p.shape[1] != 2 or p.shape[0] < 3:
        raise ValueError('BoR generatrix must be a finite (N, 2) array of (rho, z) nodes with N >= 3.')
    if not np.all(np.isfinite(p)):
        raise ValueError('BoR generatrix coordinates must all be finite.')
    scale = max(1.0, float(np.max(np.abs(p[:, 0]))))
    if np.any(p[:, 0] < -1e-12 * scale):
        raise ValueError('BoR generatrix rho coordinates must be >= 0.')
    p = p.copy()
    p[np.abs(p[:, 0]) <= 1e-12 * scale, 0] = 0.0
    if np.any(np.hypot(*np.diff(p, axis=0).T) <= 0):
        raise ValueError('BoR generatrix has a zero-length element.')
    return p


def mode_limits(k, rho_max, thetas, n_modes):
    """Mode cap (reference ``bor/solver.py:3968`` ``_bor_mode_limits``)."""
    th = np.atleast_1d(np.asarray(thetas, dtype=float))
    sin_max = float(np.max(np.abs(np.sin(np.radians(th)))))
    bandwidth = int(math.ceil(abs(k) * float(rho_max) * max(sin_max, 0.05)))
    if n_modes is None:
        cap = bandwidth + max(12, int(math.ceil(4.05 * bandwidth ** (1.0 / 3.0) + 2.0)))
    else:
        cap = int(n_modes)
        if cap < 0 or cap != n_modes:
            raise ValueError('n_modes must be a non-negative integer or None.')
    if np.all(np.isclose(np.mod(th, 180.0), 0.0)):
        return min(cap, 1), 1
    return cap, bandwidth


def pole_map(nodes, m):
    """Reduced functions of mode m: (red_full[2*nred] int32, red_w[2*nred] complex128).

    Interior nodes carry a t and a phi unknown.  An end node on the axis has no phi
    unknown and a t unknown only for |m| = 1, whose function also carries the phi
    component j m sign(t_rho) (a finite Cartesian current through the pole,
    reference ``bor/solver.py:2369-2440``).  An end node off the axis keeps phi, not t.
    """
    nn = len(nodes)
    rmax = max(1.0, float(np.max(nodes[:, 0])))
    on_axis = nodes[:, 0] <= 1e-12 * rmax
    t_act = np.ones(nn, bool)
    f_act = np.ones(nn, bool)
    for end in (0, nn - 1):
        if on_axis[end]:
            t_act[end] = abs(m) == 1
            f_act[end] = False
        else:
            t_act[end] = False
            f_act[end] = True
    full = np.concatenate([np.nonzero(t_act)[0], nn + np.nonzero(f_act)[0]])
    nred = len(full)
    red_full = -np.ones((nred, 2), dtype=np.int32)
    red_w = np.zeros((nred, 2), dtype=np.complex128)
    red_full[:, 0] = full
    red_w[:, 0] = 1.0
    if abs(m) == 1:
        d = np.diff(nodes, axis=0)
        for end, el in ((0, 0), (nn - 1, nn - 2)):
            if not on_axis[end]:
                continue
            r = int(np.nonzero(full == end)[0][0])
            red_full[r, 1] = nn + end
            red_w[r, 1] = 1j * m * (1.0 if d[el, 0] >= 0 else -1.0)
    return red_full.reshape(-1), red_w.reshape(-1), nred


MIRROR_NODE_TOLERANCE = 1e-9
MIRROR_ASYMMETRY_MAX = 1e-12

# The per-mode release gate (reference bor/solver.py constants, applied in bor/factor.py:302-355):
# every mode solution is refined against its full FP64 matrix while its 2-norm relative
# residual exceeds BOR_LINEAR_RESIDUAL_MAX or its normwise backward error exceeds
# BOR_LINEAR_BACKWARD_ERROR_MAX, and a backward error still above the latter is an error.
BOR_LINEAR_BACKWARD_ERROR_MAX = 1.0e-12
BOR_LINEAR_RESIDUAL_MAX = 1.0e-8
GATE_REFINEMENT_STEPS = 2
GATE_SLICES = 8  # the gate's residual: int8 slices on the tensor cores at FP64 GEMM accuracy


def solution_errors(Z, X, B, R, maxes, ctx=None, berr=None, relres=None):
    """R = B - Z X and the release measures of the solution X (rows of the (nrhs, n) device
    arrays are the right-hand sides): per-column backward error / 2-norm relative residual
    into ``berr`` / ``relres`` when given, their maxima into the 2-element float64 device
    view ``maxes`` (``grim_solution_errors``; reference bor/factor.py:289-300).  Queued on
    the handle's stream: call ``grim_synchronize`` (it reports the tensor-core error flag)
    before reading the results."""
    ctx = ctx or context()
    n, nrhs = int(B.shape[1]), int(B.shape[0])
    _lib.check(ctx.lib.grim_solution_errors(ctx.h, n, nrhs, ptr(Z), n, ptr(X), n, ptr(B), n, ptr(R), n, GATE_SLICES,
                                            ptr(berr), ptr(relres), ptr(maxes)), 'grim_solution_errors')


def release_limit(prec, tol):
    """Backward error a mode solved in ``prec`` is released at without gate refinement: the
    reference's limit for FP64, the refinement target ``tol`` (never tighter) for mixed."""
    if prec == 'double':
        return BOR_LINEAR_BACKWARD_ERROR_MAX
    return max(float(tol), BOR_LINEAR_BACKWARD_ERROR_MAX)


def gate_decision(berr, relres, limit):
    """Whether a solution with these maxima is released as it stands."""
    return bool(np.isfinite(berr) and np.isfinite(relres) and berr <= limit and relres <= BOR_LINEAR_RESIDUAL_MAX)


def refinement_continues(prev, cand):
    """The reference's stop rule (bor/factor.py:312-316): a refinement step is kept unless
    neither the relative residual nor the backward error (``(berr, relres)`` maxima) fell."""
    return not (cand[1] >= prev[1] and cand[0] >= prev[0])


def _measure_modes(Zs, Xs, B0s, ctx=None, workers=None, side=None):
    """The release measures of every mode solution, read in one go: a (count, 2) NumPy array
    of (backward error, relative residual) maxima.  With ``workers`` (and no ``ctx``) the
    modes run on that many device workers, so that one mode's residual overlaps the next
    one's; ``side`` (a callable taking a handle) runs beside them, first, and its result is
    returned too (None without it)."""
    count = len(Zs)
    maxes = torch.empty((count, 2), dtype=torch.float64, device='cuda')
    side_out = None
    if workers and workers > 1 and count > 1 and ctx is None:
        def job(i):
            def run():
                c = context()
                solution_errors(Zs[i], Xs[i], B0s[i], torch.empty_like(B0s[i]), maxes[i], ctx=c)
                _lib.check(c.lib.grim_synchronize(c.h), 'grim_synchronize')
            return run
        jobs = [job(i) for i in range(count)]
        if side is not None:
            jobs.insert(0, lambda: side(context()))
        res = run_pool(jobs, workers=min(int(workers), len(jobs)))
        side_out = res[0] if side is not None else None
    else:
        ctx = ctx or context()
        if side is not None:
            side_out = side(ctx)
        size = max(int(B.numel()) for B in B0s)
        scratch = torch.empty(size, dtype=torch.complex128, device='cuda')
        for i in range(count):
            R = scratch[:B0s[i].numel()].view(B0s[i].shape)
            solution_errors(Zs[i], Xs[i], B0s[i], R, maxes[i], ctx=ctx)
        _lib.check(ctx.lib.grim_synchronize(ctx.h), 'grim_synchronize')  # one wait (and error check) for all
    return maxes.cpu().numpy(), side_out


def _gate_modes(modes, Zs, Xs, B0s, precs, direct, tol, ctx=None, factors=None, measured=None):
    """The per-mode release gate over solved mode systems, in place on ``Xs``.

    ``Zs`` are the full FP64 mode matrices, ``B0s`` the right-hand sides and ``direct[i]``
    says the solution came from the FP64 LU of the full matrix (not from the mirror halves
    or a mixed-precision factor).  The residuals of all modes are measured first, then read
    in one go.  A mode that misses the gate is factored (FP64, one grouped LU of all such
    modes): a direct solution is refined from where it stands, any other one is replaced by
    the LU solution (the reference's LU fallback for a mirror factor), then up to
    GATE_REFINEMENT_STEPS refinement steps run under the reference's stop rule.  A mode
    whose backward error still exceeds BOR_LINEAR_BACKWARD_ERROR_MAX raises RuntimeError.
    Returns per-mode dicts (backward_error, relative_residual, gate_refinement_steps,
    gate_lu_fallback); with ``factors`` (a list, one entry per mode) the LU of every mode
    factored here replaces its entry.  ``measured``: the first measurements when the caller
    took them (``_measure_modes``)."""
    from ..grouped import getrf_grouped
    ctx = ctx or context()
    count = len(modes)
    if not count:
        return []
    vals = _measure_modes(Zs, Xs, B0s, ctx=ctx)[0] if measured is None else measured
    out = [{'backward_error': float(vals[i, 0]), 'relative_residual': float(vals[i, 1]), 'gate_refinement_steps': 0}
           for i in range(count)]
    bad = [i for i in range(count) if not gate_decision(vals[i, 0], vals[i, 1], release_limit(precs[i], tol))]
    if not bad:
        return out
    lus = [Zs[i].clone() for i in bad]
    ipivs, infos, _piv = getrf_grouped(lus, ctx=ctx)
    one = torch.empty(2, dtype=torch.float64, device='cuda')

    def lu_solve(j, rhs):
        n, nrhs = int(rhs.shape[1]), int(rhs.shape[0])
        _lib.check(ctx.lib.grim_zgetrs(ctx.h, n, nrhs, ptr(lus[j]), n, ptr(ipivs[j]), ptr(rhs), n), 'grim_zgetrs')

    def measure(i, X, R):
        solution_errors(Zs[i], X, B0s[i], R, one, ctx=ctx)
        _lib.check(ctx.lib.grim_synchronize(ctx.h), 'grim_synchronize')
        b, r = one.cpu().numpy()
        return float(b), float(r)

    for j, i in enumerate(bad):
        m = modes[i]
        if infos[j]:
            raise RuntimeError(f'BoR mode m={m} LU factorization failed (info={infos[j]}).')
        if not direct[i]:
            out[i]['gate_lu_fallback'] = ('mirror' if precs[i] == 'double' else 'mixed') + \
                f' solution stopped at backward error {out[i]["backward_error"]:.3g}'
            Xs[i].copy_(B0s[i])
            lu_solve(j, Xs[i])
        R, Rc = torch.empty_like(B0s[i]), torch.empty_like(B0s[i])
        cur = measure(i, Xs[i], R)  # R: the residual of the current solution
        for _step in range(GATE_REFINEMENT_STEPS):
            if cur[0] <= BOR_LINEAR_BACKWARD_ERROR_MAX and cur[1] <= BOR_LINEAR_RESIDUAL_MAX:
                break
            cand = R.clone()
            lu_solve(j, cand)
            cand += Xs[i]
            new = measure(i, cand, Rc)
            if not refinement_continues(cur, new):
                break
            Xs[i].copy_(cand)
            R, Rc = Rc, R
            cur = new
            out[i]['gate_refinement_steps'] += 1
        out[i]['backward_error'], out[i]['relative_residual'] = cur
        if not (np.isfinite(cur[0]) and np.isfinite(cur[1])) or cur[0] > BOR_LINEAR_BACKWARD_ERROR_MAX:
            raise RuntimeError(f'BoR mode m={m} normwise linear backward error {cur[0]} exceeds the release limit '
                               f'{BOR_LINEAR_BACKWARD_ERROR_MAX}.')
        if factors is not None:
            factors[i] = {'halves': None, 'lu': [lus[j]], 'ipiv': [ipivs[j]]}
    return out


# The per-mode condition gate (reference bor/solver.py BOR_CONDITION_EST_MAX, applied by
# bor/factor.py:205-229 whenever the public solve_bor runs, monitor_cond=True there).
BOR_CONDITION_EST_MAX = 1.0e12


def condition_estimates(Zs, factors, ctx=None, read=True):
    """1-norm condition estimates ||Z||_1 est(||inv(Z)||_1) of factored mode systems, all in
    one launch (``grim_zcond1_factored``: LAPACK zgecon's estimator on the device).
    ``factors[i]``: {'halves': None or the mirror map, 'lu': [LU] or [even, odd],
    'ipiv': [...]}; complex64 factors (mixed precision) are read as such.  Returns a float64
    NumPy array (NaN for a system holding a NaN, inf where zgecon's rcond is 0); with
    ``read=False`` the float64 device tensor, not waited for."""
    ctx = ctx or context()
    count = len(Zs)
    if not count:
        return np.zeros(0)
    arr = (_lib.GrimCondSystem * count)()
    for q, Z, f in zip(arr, Zs, factors):
        n = int(Z.shape[0])
        q.n, q.A, q.lda = n, Z.data_ptr(), n
        c64 = 0
        for h, lu in enumerate(f['lu']):
            q.lu[h] = lu.data_ptr()
            q.ldlu[h] = int(lu.shape[0])
            c64 |= int(lu.dtype == torch.complex64) << h
        q.lu_complex64 = c64
        mp = f['halves']
        if mp is not None:
            q.halves = 1
            q.ipiv[0], q.ipiv[1] = f['ipiv'][0].data_ptr(), f['ipiv'][1].data_ptr()
            q.k, q.nfe, q.nfo = int(mp['k']), int(mp['nfe']), int(mp['nfo'])
            q.p1, q.p2, q.s = mp['p1'].data_ptr(), mp['p2'].data_ptr(), mp['s'].data_ptr()
            q.fe, q.fo = mp['fe'].data_ptr(), mp['fo'].data_ptr()
    cond = torch.empty(count, dtype=torch.float64, device='cuda')
    _lib.check(ctx.lib.grim_zcond1_factored(ctx.h, count, ctypes.byref(arr), ptr(cond)), 'grim_zcond1_factored')
    return cond.cpu().numpy() if read else cond


def condition_gate(modes, conds):
    """The reference's release test of the mode condition estimates (bor/factor.py:224-229)."""
    for m, c in zip(modes, conds):
        if not (np.isfinite(c) and c > 0.0):
            raise RuntimeError(f'BoR mode m={m} condition estimation failed.')
        if c > BOR_CONDITION_EST_MAX:
            raise RuntimeError(f'BoR mode m={m} estimated 1-norm condition {c} exceeds the release limit '
                               f'{BOR_CONDITION_EST_MAX}.')


def mirror_map(nodes, m):
    """(target, sign) of the reduced unknowns of mode m when the generatrix is symmetric about
    a plane normal to the axis, else None (reference ``bor/solver.py:3856`` ``mirror_map``):
    the reflection z -> 2 z0 - z maps node i to node Nn - 1 - i, a reduced unknown to the same
    component of the mirrored node, J_t with sign -1 (the tangent reverses) and J_phi with +1
    (an |m| = 1 pole unknown carries its tied phi component along)."""
    nodes = np.asarray(nodes, dtype=np.float64)
    nn = len(nodes)
    size = float(max(np.ptp(nodes[:, 1]), np.max(np.abs(nodes[:, 0])), 1e-300))
    z0 = 0.5 * (nodes[0, 1] + nodes[-1, 1])
    reflected = np.column_stack([nodes[::-1, 0], 2.0 * z0 - nodes[::-1, 1]])
    if nn < 4 or float(np.max(np.abs(reflected - nodes))) > MIRROR_NODE_TOLERANCE * size:
        return None
    if (nodes[0, 0] == 0.0) != (nodes[-1, 0] == 0.0):
        return None
    rf, _rw, nred = pole_map(nodes, m)
    prim = rf.reshape(-1, 2)[:, 0]
    node, comp = prim % nn, prim // nn
    lookup = np.full(2 * nn, -1, dtype=np.int64)
    lookup[prim] = np.arange(nred)
    target = lookup[comp * nn + (nn - 1 - node)]
    if np.any(target < 0):
        return None
    return target.astype(np.int32), np.where(comp == 0, -1.0, 1.0)


def mirror_parts(target, sign):
    """Pairs (p1 < p2 = target[p1], s = sign[p2]) and fixed unknowns (fe: sign +1, fo: -1)."""
    idx = np.arange(len(target))
    paired = idx < target
    p1 = idx[paired].astype(np.int32)
    p2 = target[paired].astype(np.int32)
    fixed = idx == target
    return p1, p2, sign[p2].astype(np.float64), idx[fixed & (sign > 0)].astype(np.int32), \
        idx[fixed & (sign < 0)].astype(np.int32)


def far_points(nodes):
    x, w = np.polynomial.legendre.leggauss(FAR_ORDER)
    s = 0.5 * (x + 1.0)
    r0, r1 = nodes[:-1], nodes[1:]
    pts = r0[:, None, :] + s[None, :, None] * (r1 - r0)[:, None, :]
    return pts.reshape(-1, 2)


_RULES = None


def _near_rules():
    global _RULES
    if _RULES is None:
        _RULES = near_rules()
    return _RULES


class BorDevice:
    """Device-resident generatrix, moments and per-mode maps of one (body, k).

    ``alpha`` = 1: the EFIE; 0 < alpha < 1: the CFIE alpha EFIE + (1 - alpha) eta0 MFIE
    (the reference's closed-body default, alpha = 0.5); 0: the MFIE alone."""

    def __init__(self, points, k, mmax, ctx=None, alpha=1.0):
        self.ctx = ctx or context()
        self.nodes = validate_generatrix(points)
        self.k = float(k)
        self.mmax = int(mmax)
        self.alpha = float(alpha)
        if not 0.0 <= self.alpha <= 1.0:
            raise ValueError('alpha must lie in [0, 1]')
        self.ne = len(self.nodes) - 1
        self.nodes_dev = torch.from_numpy(np.ascontiguousarray(self.nodes.reshape(-1))).to('cuda')
        size = int(self.ctx.lib.grim_bor_moments_size(self.ne, self.mmax))
        self.mom = torch.empty(size // 16, dtype=torch.complex128, device='cuda')
        self.momk = None
        if self.alpha < 1.0:
            size = int(self.ctx.lib.grim_bor_mfie_moments_size(self.ne, self.mmax))
            self.momk = torch.empty(size // 16, dtype=torch.complex128, device='cuda')
        self.cls = np.ascontiguousarray(pair_classes(self.nodes))
        # far pairs size their own sample counts (at most MAX_NXI); no table is staged
        self.nxi = MAX_NXI
        rule, starts = _near_rules()
        _lib.check(self.ctx.lib.grim_bor_moments(self.ctx.h, self.ne, ptr(self.nodes_dev), self.k, self.mmax, self.nxi,
                                                 self.cls.ctypes.data, len(rule), rule.ctypes.data,
                                                 starts.ctypes.data, ptr(self.mom),
                                                 None if self.momk is None else ptr(self.momk)),
                   'grim_bor_moments')
        self._maps = {}

    def mode_map(self, m):
        key = m if abs(m) == 1 else (0 if m == 0 else 2)
        if key not in self._maps:
            rf, rw, nred = pole_map(self.nodes, m)
            self._maps[key] = (torch.from_numpy(rf).to('cuda'), torch.from_numpy(rw).to('cuda'), nred)
        return self._maps[key]

    def mirror(self, m):
        """Device arrays of mode m's mirror map (``mirror_map``) or None."""
        key = ('mirror', m if abs(m) == 1 else (0 if m == 0 else 2))
        if key not in self._maps:
            mp = mirror_map(self.nodes, m)
            if mp is None:
                self._maps[key] = None
            else:
                target, sign = mp
                p1, p2, sg, fe, fo = mirror_parts(target, sign)
                d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to('cuda')
                self._maps[key] = dict(target=d(target), sign=d(sign), p1=d(p1), p2=d(p2), s=d(sg), fe=d(fe),
                                       fo=d(fo), k=len(p1), nfe=len(fe), nfo=len(fo))
        return self._maps[key]

    def matrix(self, m, ctx=None):
        ctx = ctx or self.ctx
        rf, rw, nred = self.mode_map(m)
        Z = torch.empty((nred, nred), dtype=torch.complex128, device='cuda')
        _lib.check(ctx.lib.grim_bor_assemble(ctx.h, self.ne, ptr(self.nodes_dev), self.k, self.mmax, m,
                                             ptr(self.mom), None if self.momk is None else ptr(self.momk),
                                             self.alpha, nred, ptr(rf), ptr(rw), ptr(Z), nred),
                   'grim_bor_assemble')
        return Z

    def excitation(self, m, th_dev, far, ctx=None):
        ctx = ctx or self.ctx
        rf, rw, nred = self.mode_map(m)
        nth = int(th_dev.numel())
        V = torch.empty((2 * nth, nred), dtype=torch.complex128, device='cuda')
        _lib.check(ctx.lib.grim_bor_excitation(ctx.h, self.ne, ptr(self.nodes_dev), self.k, m, nth,
                                               ptr(th_dev), int(far), self.alpha, nred, ptr(rf), ptr(rw), ptr(V),
                                               nred),
                   'grim_bor_excitation')
        return V


# Mixed precision pays on a mode system only when its LU dominates and complex64 can resolve
# it: measured on the 400-segment ogive (k rho_max = 25, mode orders ~800, halves ~400), the
# complex64 refinement stalls for every |m| >= 18 = 0.72 k rho_max (their FP64 re-solve then
# doubles the work), and below that the complex64 grouped LU with its refinement takes longer
# than the FP64 LU of the same small systems (64 ms against 24 ms for all 41 modes).  So a
# mixed-precision request solves a mode in complex64 with FP64 refinement only when its
# system has at least MIXED_MIN_ORDER unknowns and |m| < MIXED_MODE_FRACTION k rho_max; the
# others are solved in FP64 (the mixed -> double ladder still guards the rest).
MIXED_MIN_ORDER = 1536
MIXED_MODE_FRACTION = 0.7


def mode_precision(dev, m, order, precision):
    """The precision one mode system is solved in under the request's ``precision``."""
    if precision != 'mixed':
        return precision
    krho = dev.k * float(np.max(dev.nodes[:, 0]))
    if order < MIXED_MIN_ORDER or abs(m) >= MIXED_MODE_FRACTION * krho:
        return 'double'
    return 'mixed'


def _factor_solve(Z, V, precision, tol, ctx):
    """LU of the mode matrix Z (complex64 with FP64 refinement for 'mixed', else complex128)
    and the solve of V in place; returns (solve telemetry, factor for condition_estimates).
    A mixed refinement that stalls raises GrimNotConverged."""
    from ..grouped import refine_factored
    n, nrhs = int(Z.shape[0]), int(V.shape[0])
    ipiv = torch.empty(n, dtype=torch.int32, device='cuda')
    info = ctypes.c_int(0)
    if precision == 'mixed':
        lu = Z.to(torch.complex64, copy=True)
        _lib.check(ctx.lib.grim_cgetrf(ctx.h, n, ptr(lu), n, ptr(ipiv), ctypes.byref(info)), 'grim_cgetrf')
    else:
        lu = Z.clone()
        _lib.check(ctx.lib.grim_zgetrf(ctx.h, n, ptr(lu), n, ptr(ipiv), ctypes.byref(info)), 'grim_zgetrf')
    if info.value:
        raise _lib.GrimError(_lib.GRIM_ERR_SINGULAR, f'BoR mode matrix is exactly singular (info={info.value})')
    if precision == 'mixed':
        st = refine_factored(Z, lu, ipiv, V, tol, stop='berr', ctx=ctx)
    else:
        _lib.check(ctx.lib.grim_zgetrs(ctx.h, n, nrhs, ptr(lu), n, ptr(ipiv), ptr(V), n), 'grim_zgetrs')
        st = {'precision_mode': _lib.PREC_FP64}
    return st, {'halves': None, 'lu': [lu], 'ipiv': [ipiv]}


def _solve_mode(dev, m, th, precision, tol, ctx=None, monitor_cond=True):
    """One Fourier mode on ``ctx`` (default: the current device worker): assemble, excite,
    factor, solve and project.  The release measures (and with ``monitor_cond`` the
    condition estimate) are queued on the device, not read: returns (this mode's far-field
    contribution [2 nth], telemetry, pending device results for ``_finish_modes``)."""
    ctx = ctx or context()
    Z = dev.matrix(m, ctx=ctx)
    V = dev.excitation(m, th, far=False, ctx=ctx)
    W = dev.excitation(m, th, far=True, ctx=ctx)
    tele = {'fp64_fallback': False}
    if tol is None:
        tol = ops2d.MIXED_RCS_TOL  # an RCS solve: the same refinement target as the 2-D RCS path
    precision = mode_precision(dev, m, int(Z.shape[0]), precision)
    V0 = V.clone()
    try:
        st, factor = _factor_solve(Z, V, precision, tol, ctx)
    except _lib.GrimNotConverged:
        # ill-conditioned mode: the reference's ladder falls back to the double LU
        tele['fp64_fallback'] = True
        V.copy_(V0)
        precision = 'double'
        st, factor = _factor_solve(Z, V, precision, tol, ctx)
    tele['refinement_steps'] = int(st.get('refinement_steps', 0))
    pending = {'precision': precision, 'maxes': torch.empty(2, dtype=torch.float64, device='cuda'), 'cond': None}
    solution_errors(Z, V, V0, torch.empty_like(V0), pending['maxes'], ctx=ctx)
    if monitor_cond:
        pending['cond'] = condition_estimates([Z], [factor], ctx=ctx, read=False)
    nth = int(th.numel())
    part = torch.zeros(2 * nth, dtype=torch.complex128, device='cuda')
    nred = int(Z.shape[0])
    _lib.check(ctx.lib.grim_bor_farfield_accumulate(ctx.h, nred, 2 * nth, ptr(W), nred, ptr(V), nred, ptr(part)),
               'grim_bor_farfield_accumulate')
    return part, tele, pending


def _pool_mode(dev, m, th, precision, tol, monitor_cond):
    """``_solve_mode`` on a device worker, its handle's tensor-core error flag checked."""
    out = _solve_mode(dev, m, th, precision, tol, monitor_cond=monitor_cond)
    c = context()
    _lib.check(c.lib.grim_synchronize(c.h), 'grim_synchronize')
    return out


def _redo_mode(dev, m, th, tol, ctx, monitor_cond):
    """A mode that missed the release gate, again from its FP64 LU: assemble, factor, solve,
    then the gate's refinement (``_gate_modes``, which raises when the backward error stays
    above the limit) and, with ``monitor_cond``, the condition gate on the new factor.
    Returns (far-field contribution, gate telemetry)."""
    Z = dev.matrix(m, ctx=ctx)
    V = dev.excitation(m, th, far=False, ctx=ctx)
    W = dev.excitation(m, th, far=True, ctx=ctx)
    V0 = V.clone()
    _st, factor = _factor_solve(Z, V, 'double', tol, ctx)
    factors = [factor]
    gate = _gate_modes([m], [Z], [V], [V0], ['double'], [True], tol, ctx=ctx, factors=factors)[0]
    if monitor_cond:
        cond = condition_estimates([Z], factors, ctx=ctx)
        condition_gate([m], cond)
        gate['condition_est'] = float(cond[0])
    nth = int(th.numel())
    part = torch.zeros(2 * nth, dtype=torch.complex128, device='cuda')
    nred = int(Z.shape[0])
    _lib.check(ctx.lib.grim_bor_farfield_accumulate(ctx.h, nred, 2 * nth, ptr(W), nred, ptr(V), nred, ptr(part)),
               'grim_bor_farfield_accumulate')
    return part, gate


def _finish_modes(dev, modes, th, results, tol, ctx, monitor_cond):
    """The gates over modes solved by ``_solve_mode``: one read of every mode's queued
    condition estimate and release measures, the condition gate in mode order, then each
    mode that missed the release limits solved again from its FP64 LU with refinement
    (``_redo_mode``; a mixed solution that misses them is replaced by the LU solution, as
    the grouped path does).  Returns [(part, telemetry)]."""
    ctx = ctx or context()
    if tol is None:
        tol = ops2d.MIXED_RCS_TOL
    if not results:
        return []
    _lib.check(ctx.lib.grim_synchronize(ctx.h), 'grim_synchronize')
    vals = torch.stack([p['maxes'] for _part, _t, p in results]).cpu().numpy()
    conds = None
    if monitor_cond:
        conds = torch.cat([p['cond'] for _part, _t, p in results]).cpu().numpy()
        condition_gate(modes, conds)
    outs = []
    for i, (m, (part, tele, p)) in enumerate(zip(modes, results)):
        tele.update(backward_error=float(vals[i, 0]), relative_residual=float(vals[i, 1]), gate_refinement_steps=0)
        if conds is not None:
            tele['condition_est'] = float(conds[i])
        if not gate_decision(vals[i, 0], vals[i, 1], release_limit(p['precision'], tol)):
            part, gate = _redo_mode(dev, m, th, tol, ctx, monitor_cond)
            if p['precision'] != 'double':
                gate['gate_lu_fallback'] = f'mixed solution stopped at backward error {vals[i, 0]:.3g}'
            tele.update(gate)
        outs.append((part, tele))
    return outs


def _mirror_modes(dev, modes, Zs):
    """Indices of the modes whose matrices are mirror-symmetric to MIRROR_ASYMMETRY_MAX
    (relative to their largest entry): max |Z - R Z R| on the device, read in one go."""
    ctx = context()
    checks = []
    for i, (m, Z) in enumerate(zip(modes, Zs)):
        mp = dev.mirror(m)
        if mp is None:
            continue
        out = torch.empty(2, dtype=torch.float64, device='cuda')
        n = int(Z.shape[0])
        _lib.check(ctx.lib.grim_bor_mirror_asymmetry(ctx.h, n, ptr(Z), n, ptr(mp['target']), ptr(mp['sign']),
                                                     ptr(out)), 'grim_bor_mirror_asymmetry')
        checks.append((i, out))
    if not checks:
        return []
    vals = torch.stack([o for _i, o in checks]).cpu().numpy()
    return [i for (i, _o), (d, a) in zip(checks, vals) if np.isfinite(d) and d <= MIRROR_ASYMMETRY_MAX * a]


def _solve_mirror_grouped(dev, modes, Zs, Vs, workers, precision='double', tol=None, keep_factors=False):
    """Solves of mirror-symmetric mode systems through their even and odd halves (reference
    ``bor/factor.py:37`` ``MirrorSplit``): the halves of every mode (FP64) and the split
    right-hand sides, one grouped solve of all halves (``grouped.solve_grouped``: a quarter
    of the LU work; mixed: complex64 factors refined against the FP64 halves, a half whose
    refinement stalls re-solved in FP64), then the join.  The modes were checked symmetric
    to MIRROR_ASYMMETRY_MAX, so the halves are the system itself to rounding; the release
    gate (``_gate_modes``) then checks every joined solution against the full matrix and
    replaces one that misses it by the LU solution.  With ``keep_factors`` returns
    (telemetry, factors): per mode the halves' LUs for ``condition_estimates``."""
    from ..grouped import solve_grouped
    ctx = context()
    halves, rhs, args_of = [], [], []
    for m, Z, V in zip(modes, Zs, Vs):
        mp = dev.mirror(m)
        n = int(Z.shape[0])
        nrhs = int(V.shape[0])
        ke, ko = mp['k'] + mp['nfe'], mp['k'] + mp['nfo']
        He = torch.empty((ke, ke), dtype=torch.complex128, device='cuda')
        Ho = torch.empty((ko, ko), dtype=torch.complex128, device='cuda')
        _lib.check(ctx.lib.grim_bor_mirror_halves(ctx.h, n, ptr(Z), n, mp['k'], ptr(mp['p1']), ptr(mp['p2']),
                                                  ptr(mp['s']), mp['nfe'], ptr(mp['fe']), mp['nfo'], ptr(mp['fo']),
                                                  ptr(He), ptr(Ho)), 'grim_bor_mirror_halves')
        args = (mp['k'], ptr(mp['p1']), ptr(mp['p2']), ptr(mp['s']), mp['nfe'], ptr(mp['fe']), mp['nfo'], ptr(mp['fo']))
        Be = torch.empty((nrhs, ke), dtype=torch.complex128, device='cuda')
        Bo = torch.empty((nrhs, ko), dtype=torch.complex128, device='cuda')
        _lib.check(ctx.lib.grim_bor_mirror_split(ctx.h, nrhs, ptr(V), n, *args, ptr(Be), ptr(Bo)),
                   'grim_bor_mirror_split')
        halves += [He, Ho]
        rhs += [Be, Bo]
        args_of.append((args, nrhs, n, ke, ko))
    mixed = precision == 'mixed'
    rhs0 = [b.clone() for b in rhs] if mixed else None
    sts = solve_grouped(halves, rhs, precision=precision, tol=tol, stop='berr', workers=workers,
                        keep_factors=keep_factors)
    stalled = [i for i, st in enumerate(sts) if st.get('not_converged')]
    if stalled:
        redo = solve_grouped([halves[i] for i in stalled], [rhs0[i] for i in stalled], precision='double',
                             workers=workers, keep_factors=keep_factors)
        for i, st in zip(stalled, redo):
            sts[i] = dict(st, fp64_fallback=True)
            rhs[i] = rhs0[i]
    facs = [(st.pop('lu', None), st.pop('ipiv', None)) for st in sts]
    out, factors = [], []
    for j, (args, nrhs, n, ke, ko) in enumerate(args_of):
        _lib.check(ctx.lib.grim_bor_mirror_join(ctx.h, nrhs, ptr(rhs[2 * j]), ptr(rhs[2 * j + 1]), *args, ptr(Vs[j]), n),
                   'grim_bor_mirror_join')
        se, so = sts[2 * j], sts[2 * j + 1]
        out.append({'precision_mode': se.get('precision_mode', _lib.PREC_FP64),
                    'pivoted_panels': se.get('pivoted_panels', 0) + so.get('pivoted_panels', 0), 'grouped': True,
                    'mirror_halves': [ke, ko], 'fp64_fallback': bool(se.get('fp64_fallback') or so.get('fp64_fallback')),
                    'refinement_steps': max(int(se.get('refinement_steps', 0)), int(so.get('refinement_steps', 0)))})
        if keep_factors:
            (lue, pe), (luo, po) = facs[2 * j], facs[2 * j + 1]
            factors.append({'halves': dev.mirror(modes[j]), 'lu': [lue, luo], 'ipiv': [pe, po]})
    return (out, factors) if keep_factors else out


def _solve_modes_grouped(dev, modes, th, precision, tol, workers, monitor_cond=True):
    """All mode systems through one grouped LU (``grouped.solve_grouped``): assembly and
    excitations on the worker pool, one grouped factorization of every mode matrix, then
    the per-mode solves / refinement on the pool and the far-field projections here.  A
    mode whose refinement stalls is re-solved in FP64 (the reference's ladder).  With
    ``monitor_cond`` (the reference's public solve_bor) the factors are kept and every
    mode's condition estimate is taken and gated before the release gate, as the
    reference's ModalFactor does at construction; a mode the release gate refactors is
    estimated again from its new LU."""
    from ..grouped import solve_grouped

    def prep(m):
        def run():
            c = context()
            return dev.matrix(m, ctx=c), dev.excitation(m, th, far=False, ctx=c), dev.excitation(m, th, far=True, ctx=c)
        return run

    import time
    t0 = time.perf_counter()
    parts = run_pool([prep(m) for m in modes], workers=workers)
    Zs = [p[0] for p in parts]
    Vs = [p[1] for p in parts]
    V0s = [v.clone() for v in Vs]
    if tol is None:
        tol = ops2d.MIXED_RCS_TOL
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    mirrored = set(_mirror_modes(dev, modes, Zs))
    sts = [None] * len(modes)
    factors = [None] * len(modes)
    precs = [mode_precision(dev, m, int(Zs[i].shape[0]), precision) for i, m in enumerate(modes)]
    for prec in ('double', 'mixed'):
        mine = [i for i in range(len(modes)) if precs[i] == prec]
        mir = [i for i in mine if i in mirrored]
        if mir:
            res = _solve_mirror_grouped(dev, [modes[i] for i in mir], [Zs[i] for i in mir], [Vs[i] for i in mir],
                                        workers, precision=prec, tol=tol, keep_factors=monitor_cond)
            outs_m, facs = res if monitor_cond else (res, [None] * len(mir))
            for i, st, f in zip(mir, outs_m, facs):
                sts[i], factors[i] = st, f
        rest = [i for i in mine if i not in mirrored]
        if rest:
            for i, st in zip(rest, solve_grouped([Zs[i] for i in rest], [Vs[i] for i in rest], precision=prec,
                                                 tol=tol, stop='berr', workers=workers, keep_factors=monitor_cond)):
                sts[i] = st
                factors[i] = {'halves': None, 'lu': [st.pop('lu', None)], 'ipiv': [st.pop('ipiv', None)]}
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    # stalled refinements (ill-conditioned modes): the reference's ladder to the double LU,
    # here one grouped FP64 factorization of all of them (into copies: V0s stay the
    # right-hand sides of the release gate)
    stalled = [i for i, st in enumerate(sts) if st.get('not_converged')]
    if stalled:
        xs = [V0s[i].clone() for i in stalled]
        redo = solve_grouped([Zs[i] for i in stalled], xs, precision='double', workers=workers,
                             keep_factors=monitor_cond)
        for i, st, x in zip(stalled, redo, xs):
            factors[i] = {'halves': None, 'lu': [st.pop('lu', None)], 'ipiv': [st.pop('ipiv', None)]}
            sts[i] = dict(st, fp64_fallback=True)
            Vs[i] = x
    torch.cuda.synchronize()
    t3 = time.perf_counter()
    # the condition estimates (one launch, a CTA per mode) run beside the release measures
    # of every mode on the worker pool; the condition gate is applied first, as the
    # reference's factor construction does
    side = (lambda c: condition_estimates(Zs, factors, ctx=c, read=False)) if monitor_cond else None
    vals, cond_dev = _measure_modes(Zs, Vs, V0s, workers=workers, side=side)
    conds = None
    if monitor_cond:
        conds = cond_dev.cpu().numpy()
        condition_gate(modes, conds)
    t4 = time.perf_counter()
    # the release gate against every full mode matrix: a solution from the FP64 LU of the
    # full matrix is direct; mirror halves and mixed factors are not
    fell_back = [bool(st.get('fp64_fallback')) for st in sts]
    eff = ['double' if fb and i not in mirrored else precs[i] for i, fb in enumerate(fell_back)]
    direct = [i not in mirrored and eff[i] == 'double' for i in range(len(modes))]
    gate = _gate_modes(modes, Zs, Vs, V0s, eff, direct, tol, factors=factors if monitor_cond else None,
                       measured=vals)
    redone = [i for i in range(len(modes)) if gate[i].get('gate_lu_fallback')]
    if monitor_cond and redone:
        again = condition_estimates([Zs[i] for i in redone], [factors[i] for i in redone])
        condition_gate([modes[i] for i in redone], again)
        conds[redone] = again
    torch.cuda.synchronize()
    stage = {'assembly': t1 - t0, 'grouped_factor_and_solves': t2 - t1, 'fp64_fallbacks': t3 - t2,
             'condition_and_release_measures': t4 - t3, 'release_gate': time.perf_counter() - t4}
    ctx = context()
    nth = int(th.numel())
    outs = []
    for i, st in enumerate(sts):
        tele = {'fp64_fallback': fell_back[i], 'grouped': True, 'stage_seconds': stage, **gate[i]}
        if conds is not None:
            tele['condition_est'] = float(conds[i])
        V = Vs[i]
        tele['refinement_steps'] = int(st.get('refinement_steps', 0))
        part = torch.zeros(2 * nth, dtype=torch.complex128, device='cuda')
        nred = int(Zs[i].shape[0])
        _lib.check(ctx.lib.grim_bor_farfield_accumulate(ctx.h, nred, 2 * nth, ptr(parts[i][2]), nred, ptr(V), nred,
                                                        ptr(part)), 'grim_bor_farfield_accumulate')
        outs.append((part, tele))
    return outs


def solve_bor_device(points, k, thetas_deg, mmax, precision='double', tol=None, ctx=None, workers=None,
                     signed_mode_symmetry=True, grouped=True, mode_tol=None, tail_start=0, alpha=1.0,
                     monitor_cond=True):
    """Device path: returns (F[2 nth] complex128 on the host, telemetry).

    The modal moments are built once; the per-mode systems are independent and run on the
    device worker pool (``GRIM_SWEEP_WORKERS`` workers), each contributing its own
    far-field vector; the contributions are summed in mode order, so the result does not
    depend on the scheduling.  With ``signed_mode_symmetry`` (the reference's setting in
    every solve_bor path, ``bor/solver.py:2972,3061``) only m = 0..mmax are solved and
    m > 0 counts twice: for the co-polarised monostatic far field the +m and -m
    contributions are identical (equal to the last bit in the oracle, for the sphere and
    the ogive).  With an explicit ``ctx`` (a serving slot) the modes run in turn on that
    handle.  ``alpha`` selects the formulation (``BorDevice``).  With ``grouped`` (default) the mode systems are factored together by one
    grouped LU (``grouped.py``); otherwise each mode is factored on its own worker.  With
    ``mode_tol`` the modal sum stops at the reference's adaptive tail (two consecutive
    modes at or above ``tail_start`` below the tolerance; ``_adaptive_tail``); all modes up
    to ``mmax`` are solved together first, so the truncation decides only the sum.  Every
    mode passes the reference's release gates: its condition estimate (``monitor_cond``,
    on in the reference's public solve_bor) and its backward error against the full matrix.
    """
    from ..twod.solver import sweep_workers
    import time
    tm = time.perf_counter()
    dev = BorDevice(points, k, mmax, ctx=ctx, alpha=alpha)
    for m in (0, 1, -1, 2):
        dev.mode_map(m)  # build the shared pole maps before the workers read them
    torch.cuda.synchronize()
    t_moments = time.perf_counter() - tm
    th = torch.as_tensor(np.asarray(thetas_deg, dtype=np.float64), device='cuda')
    modes = list(range(0, mmax + 1)) if signed_mode_symmetry else list(range(-mmax, mmax + 1))

    def solve_local(idx):
        sub = [modes[i] for i in idx]
        if not sub:
            return []
        if ctx is not None:
            res = [_solve_mode(dev, m, th, precision, tol, ctx=ctx, monitor_cond=monitor_cond) for m in sub]
            return _finish_modes(dev, sub, th, res, tol, ctx, monitor_cond)
        if grouped:
            return _solve_modes_grouped(dev, sub, th, precision, tol,
                                        sweep_workers(len(sub)) if workers is None else workers,
                                        monitor_cond=monitor_cond)
        jobs = [(lambda m=m: _pool_mode(dev, m, th, precision, tol, monitor_cond)) for m in sub]
        res = run_pool(jobs, workers=sweep_workers(len(jobs)) if workers is None else workers)
        return _finish_modes(dev, sub, th, res, tol, None, monitor_cond)

    shard, group = requested_shard_group()
    if shard and ctx is None:
        # every rank holds the moments; the mode systems are split over the ranks (equal
        # cost per mode) and their far-field contributions gathered on the host
        def run_local(idx):
            return [(part.cpu().numpy(), {kk: vv for kk, vv in t.items() if not hasattr(vv, 'cpu')})
                    for part, t in solve_local(idx)]
        outs = [(torch.as_tensor(part, device='cuda'), t)
                for part, t in sharding.run_sharded([1.0] * len(modes), run_local, group)]
    else:
        outs = solve_local(range(len(modes)))
    amp = torch.zeros(2 * int(th.numel()), dtype=torch.complex128, device='cuda')
    modes_used, tail = mmax, None
    if mode_tol is not None and signed_mode_symmetry:
        modes_used, tail = _adaptive_tail([(2.0 if m > 0 else 1.0) * part for m, (part, _t) in zip(modes, outs)],
                                          float(mode_tol), int(tail_start))
    for m, (part, _t) in zip(modes, outs):
        if signed_mode_symmetry and abs(m) > modes_used:
            continue
        if signed_mode_symmetry and m > 0:
            amp += 2.0 * part
        else:
            amp += part
    tele = {'modes': 2 * mmax + 1, 'mode_systems_solved': len(modes),
            'max_backward_error': max(t['backward_error'] for _p, t in outs),
            'max_relative_residual': max(t['relative_residual'] for _p, t in outs),
            'backward_error_max': BOR_LINEAR_BACKWARD_ERROR_MAX, 'residual_norm_refinement_advisory': BOR_LINEAR_RESIDUAL_MAX,
            'refinement_steps': max(t['refinement_steps'] for _p, t in outs)}
    tele['linear_refinement_steps'] = int(sum(t.get('gate_refinement_steps', 0) for _p, t in outs))
    tele['condition_est_computed'] = bool(monitor_cond)
    tele['condition_est_limit'] = BOR_CONDITION_EST_MAX
    if monitor_cond:
        conds = [t['condition_est'] for _p, t in outs]
        tele['condition_est_method'] = 'lapack_gecon_1norm'
        tele['max_cond'] = float(max(conds))
        tele['median_cond'] = float(np.median(conds))
    gated = [m for m, (_p, t) in zip(modes, outs) if t.get('gate_refinement_steps') or t.get('gate_lu_fallback')]
    if gated:
        tele['gate_refined_modes'] = gated
        tele['gate_lu_fallback_modes'] = [m for m, (_p, t) in zip(modes, outs) if t.get('gate_lu_fallback')]
    fallbacks = [m for m, (_p, t) in zip(modes, outs) if t['fp64_fallback']]
    if fallbacks:
        tele['fp64_fallback_modes'] = len(fallbacks)
        tele['fp64_fallback_mode_list'] = fallbacks
    tele['stage_seconds'] = dict(modal_moments=t_moments, **(outs[0][1].get('stage_seconds') or {}))
    F = amp.cpu().numpy() * (-1j * k * ETA0 / (4.0 * np.pi))
    tele['n_unknowns'] = 2 * (dev.ne + 1)
    tele['modes_used'] = int(modes_used)
    if tail is not None:
        tele.update(tail)
    return F, tele


def _adaptive_tail(contributions, mode_tol, tail_start):
    """The reference's modal convergence rule (``bor/solver.py:3130-3190``): accumulate the
    |m| = 0, 1, ... contributions in order; after each, the worst relative increment over
    the samples is |dF| / (|F| + mode_tol max|F|); stop once two consecutive modes at or
    above ``tail_start`` stay below ``mode_tol``.  Returns (last mode used, report)."""
    F = None
    quiet, used, rel = 0, 0, 0.0
    for am, dF in enumerate(contributions):
        d = dF.cpu().numpy()
        F = d.copy() if F is None else F + d
        fa, da = np.abs(F), np.abs(d)
        scale = max(float(np.max(fa)), 1e-300)
        eff = fa + mode_tol * scale
        rel = float(np.max(np.divide(da, eff, out=np.zeros_like(da), where=eff > 0.0)))
        used = am
        quiet = quiet + 1 if (am >= tail_start and rel < mode_tol) else 0
        if quiet >= 2:
            break
    return used, {'mode_converged': bool(quiet >= 2), 'mode_selection': 'adaptive_tail',
                  'mode_tail_start': int(tail_start), 'mode_last_relative_increment': rel}


def solve_bor(points, freq_hz, thetas_deg, formulation="auto", cfie_alpha=0.5, zs=None, n_modes=None,
              gauss_order=FAR_ORDER, mode_tol=1e-6, workers=1, progress=None, check_abort=None,
              table_precision="auto", assembly="auto", stream_budget_gb=8.0, sheet_zs=None):
    """Monostatic VV/HH RCS of a PEC BoR at aspects ``thetas_deg`` (from +z).

    Same arguments and result keys as the reference's ``solve_bor``
    (``bor/solver.py:4066``).  ``formulation``: 'auto' selects the CFIE for a closed body
    (both generatrix ends on the axis) and the EFIE otherwise, as the reference does;
    'cfie' (alpha EFIE + (1 - alpha) eta0 MFIE, ``cfie_alpha`` in (0, 1)) and 'mfie' need a
    closed body traversed from the +z pole to the -z pole; 'efie' also serves open shells.
    """
    form = str(formulation).strip().lower()
    if form not in {'auto', 'efie', 'cfie', 'mfie'}:
        raise ValueError(f"Unsupported BoR formulation '{formulation}'. Use 'auto', 'efie', 'cfie', or 'mfie'.")
    if form in {'cfie', 'auto'}:
        cfie_alpha = float(cfie_alpha)
        if not np.isfinite(cfie_alpha) or not (0.0 < cfie_alpha < 1.0):
            raise ValueError('CFIE alpha must be finite and satisfy 0 < alpha < 1.')
    if zs is not None or sheet_zs is not None:
        raise NotImplementedError('Impedance and sheet BoR models are outside the GPU PEC path.')
    if int(gauss_order) != FAR_ORDER:
        raise ValueError(f'The GPU BoR path integrates far pairs with {FAR_ORDER} Gauss points per element.')
    require_cuda()
    pts = validate_generatrix(points)
    closed = pts[0, 0] == 0.0 and pts[-1, 0] == 0.0
    if form == 'auto':
        form = 'cfie' if closed else 'efie'
    if form in {'cfie', 'mfie'}:
        if not closed:
            raise ValueError(f'{form.upper()} requires a closed BoR whose two generatrix endpoints lie on the '
                             'rotation axis; use EFIE for an intentionally open shell.')
        if not pts[0, 1] > pts[-1, 1]:
            raise ValueError('A closed BoR generatrix must be traversed from its +z axis endpoint to its -z axis '
                             'endpoint so the left-of-travel normal faces the exterior.')
    alpha = {'efie': 1.0, 'cfie': cfie_alpha, 'mfie': 0.0}[form]
    thetas = np.asarray(thetas_deg, dtype=np.float64).reshape(-1)
    if thetas.size == 0 or not np.all(np.isfinite(thetas)):
        raise ValueError('BoR aspects must be a non-empty list of finite angles.')
    k = 2.0 * math.pi * float(freq_hz) / C0
    mcap, bandwidth = mode_limits(k, float(np.max(pts[:, 0])), thetas, n_modes)
    if check_abort is not None:
        check_abort()
    F, tele = solve_bor_device(pts, k, thetas, mcap, precision=requested_precision(), mode_tol=mode_tol,
                               tail_start=bandwidth, alpha=alpha)
    nth = len(thetas)
    Fv, Fh = F[:nth], F[nth:]
    return {
        'theta_deg': thetas.tolist(),
        'sigma_vv': (4.0 * math.pi * np.abs(Fv) ** 2).tolist(),
        'sigma_hh': (4.0 * math.pi * np.abs(Fh) ** 2).tolist(),
        'amp_vv': Fv.tolist(),
        'amp_hh': Fh.tolist(),
        'modes_used': int(tele['modes_used']),
        'mode_converged': bool(tele.get('mode_converged', False)),
        'mode_cap': int(mcap),
        'n_unknowns': int(tele['n_unknowns']),
        'formulation': form,
        'boundary_model': 'pec',
        'assembly': 'gpu_moments',
        'table_precision': 'double',
        'device': context().device_name,
        'precision': requested_precision(),
        'warnings': [],
        'mode_bandwidth': int(bandwidth),
        # the reference's release statistics (bor/solver.py:3195-3240)
        'linear_residual': float(tele['max_relative_residual']),
        'linear_backward_error': float(tele['max_backward_error']),
        'linear_refinement_steps': int(tele['linear_refinement_steps']),
        'linear_residual_limit': BOR_LINEAR_RESIDUAL_MAX,
        'linear_residual_limit_kind': 'iterative_refinement_advisory',
        'linear_backward_error_limit': BOR_LINEAR_BACKWARD_ERROR_MAX,
        'condition_est_computed': True,
        'condition_est_method': 'lapack_gecon_1norm',
        'condition_est_limit': BOR_CONDITION_EST_MAX,
        'max_cond': float(tele['max_cond']),
        'median_cond': float(tele['median_cond']),
    }
