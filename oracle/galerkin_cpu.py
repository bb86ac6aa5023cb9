"""CPU timing port of the linear-Galerkin combined-field solve (TEST INFRASTRUCTURE).

Only ``bench.py``'s CPU-baseline legs import this module: it times, on the host cores,
the work of one (geometry, frequency, polarisation) solve in the reference's own 2-D
formulation, restated with NumPy / SciPy as the reference's NumPy path computes it
(``twod/operators.py:2087`` ``_assemble_multi``: far pairs by a Gauss tensor rule with
SciPy's Bessel functions, near pairs by the self / touching / adaptive / fixed rules;
``linalg/dense.py`` LAPACK LU and solve):

* ``far_rows_numpy`` / ``far_rows_compiled`` / ``near_rows`` -- the element-pair S and K'
  blocks of a set of observation element rows against every source element: far pairs
  (centre distance >= 3 max(L), no shared node) with the 8-point rule (the reference's
  order after its W floor; every far block within 1e-12 of a converged rule), vectorised
  with SciPy's Bessel functions or through the reference's own compiled ``far.c``; near
  pairs through ``oracle.galerkin2d``'s pinned rules;
* ``near_all`` -- every near pair of the contour, batched by rule (vectorised touching and
  fixed-rule pairs, close pairs refined level by level across all of them at once);
* ``time_solve`` -- one solve: the far pass (all rows, or a sample scaled to N), the near
  pass, LAPACK LU and the solve of all right-hand sides, the plane-wave loads and the far
  field.
"""
from __future__ import annotations

import time

import numpy as np
import scipy.linalg as sla
from scipy import special as sp

from . import galerkin2d as G

FAR_ORDER = 8


def _contour(drawn):
    nodes = G.drawn_to_solver_contour(drawn)
    n = len(nodes)
    a = nodes
    b = np.roll(nodes, -1, axis=0)
    d = b - a
    length = np.hypot(d[:, 0], d[:, 1])
    normal = np.stack([-d[:, 1], d[:, 0]], axis=1) / length[:, None]
    return nodes, a, b, length, normal, n


def _far_mask(centre, length, e, n):
    ratio = np.hypot(*(centre - centre[e]).T) / np.maximum(length, length[e])
    share = np.zeros(n, bool)
    share[[e, (e + 1) % n, (e - 1) % n]] = True
    return (ratio >= 3.0) & ~share, share


def far_rows_numpy(drawn, k, rows, order=FAR_ORDER):
    """Far-pair S and K' blocks of element rows ``rows``: NumPy tensor rule, SciPy Bessel."""
    nodes, a, b, length, normal, n = _contour(drawn)
    t, w = G.unit_gauss(order)
    centre = 0.5 * (a + b)
    ww = np.outer(w, w)
    bo = np.stack([1.0 - t, t], axis=1)
    out = []
    for e in rows:
        far, _share = _far_mask(centre, length, e, n)
        fi = np.flatnonzero(far)
        xo = a[e][None, :] + t[:, None] * (b[e] - a[e])[None, :]                      # (q, 2)
        ys = a[fi][:, None, :] + t[None, :, None] * (b[fi] - a[fi])[:, None, :]          # (nf, q, 2)
        diff = xo[None, :, None, :] - ys[:, None, :, :]                                  # (nf, q, q, 2)
        r = np.sqrt(np.sum(diff * diff, axis=-1))
        kr = k * r
        g = 0.25 * sp.y0(kr) + 0.25j * sp.j0(kr)
        h = 0.25 * k * sp.y1(kr) + 0.25j * k * sp.j1(kr)
        proj = -np.einsum('fpqc,c->fpq', diff, normal[e]) / r
        sc = (length[e] * length[fi])[:, None, None]
        out.append((e, np.einsum('fpq,pa,qb->fab', g * ww, bo, bo) * sc,
                    np.einsum('fpq,pa,qb->fab', h * proj * ww, bo, bo) * sc))
    return out


def far_rows_compiled(drawn, k, rows, far_block_fn, table, order=FAR_ORDER):
    """Far-pair S, K' and mirrored K blocks of element rows ``rows`` against the elements
    after them (the mirrored K gives the transposed pairs, as the reference's symmetric tile
    traversal does) through a compiled ``ghost_far_block`` (``twod/assembly/native/far.c:193``,
    the reference's own C far pass;
    ``far_block_fn(mb, nb, q, obs_pts, src_pts, qw, phi, obs_norm, src_norm, far, table)``
    returns its three accumulators)."""
    nodes, a, b, length, normal, n = _contour(drawn)
    x, w = np.polynomial.legendre.leggauss(order)
    t = 0.5 * (x + 1.0)
    pts = np.ascontiguousarray(a[:, None, :] + t[None, :, None] * (b - a)[:, None, :])
    qw = np.ascontiguousarray(0.5 * w)
    phi = np.ascontiguousarray(np.stack([1.0 - t, t], axis=1))
    centre = 0.5 * (a + b)
    rows = np.asarray(list(rows), dtype=np.int64)
    far = np.zeros((len(rows), n), np.uint8)
    for i, e in enumerate(rows):
        far[i] = _far_mask(centre, length, e, n)[0]
        far[i, :e + 1] = 0  # the pairs f > e: the kernel's mirrored K gives (f, e) from the same points
    return far_block_fn(len(rows), n, order, np.ascontiguousarray(pts[rows]), pts, qw, phi,
                        np.ascontiguousarray(normal[rows]), np.ascontiguousarray(normal), far, table)


def near_rows(drawn, k, rows):
    """Near-pair (self, touching, adaptive and fixed-rule) S and K' blocks of element rows
    ``rows`` through the oracle's rules: [(e, f, S, K')]."""
    nodes, a, b, length, normal, n = _contour(drawn)
    centre = 0.5 * (a + b)
    ends = [(a[i], b[i]) for i in range(n)]
    out = []
    for e in rows:
        far, share = _far_mask(centre, length, e, n)
        for f in np.flatnonzero(~far):
            if f == e:
                out.append((e, f, G.self_block(length[e], k), np.zeros((2, 2), complex)))
            elif share[f]:
                obs_start = f == (e - 1) % n
                out.append((e, f, *G.touching_blocks(ends[e], ends[f], normal[e], normal[f], obs_start,
                                                     not obs_start, k, True)))
            elif G.needs_adaptive(ends[e], ends[f]):
                out.append((e, f, *G.adaptive_blocks(ends[e], ends[f], normal[e], normal[f], k, True)))
            else:
                out.append((e, f, *G.box_blocks(ends[e], ends[f], normal[e], normal[f], k, True)))
    return out


def _hankel_pair(k, r):
    """(j/4) H0^(2)(k r) and (j/4) k H1^(2)(k r) with the oracle's floors (r >= 1e-12, k r >= 1e-12)."""
    x = np.maximum(k * np.maximum(r, G.EPS), 1e-12)
    return 0.25 * sp.y0(x) + 0.25j * sp.j0(x), 0.25 * k * sp.y1(x) + 0.25j * k * sp.j1(x)


def _blocks(w, g, dk, xo, xs, scale):
    """sum_q w g phi_a(xo) phi_b(xs) (and the same for dk) times scale, per pair."""
    bo = np.stack([1.0 - xo, xo], axis=-1)
    bs = np.stack([1.0 - xs, xs], axis=-1)
    s_blk = np.einsum('pq,pqa,pqb->pab', w * g, bo, bs) * scale[:, None, None]
    k_blk = np.einsum('pq,pqa,pqb->pab', w * dk, bo, bs) * scale[:, None, None]
    return s_blk, k_blk


def _boxes(a, b, normal, k, eo, es, oa, ob, sa, sb, order=G.BOX_ORDER):
    """S and K' (observation normal) of the sub-interval boxes [oa, ob] x [sa, sb] of pairs
    (eo, es) in the parent hat bases, the 16-point tensor rule, all boxes at once."""
    t, w = G.unit_gauss(order)
    ho, hs = ob - oa, sb - sa
    xo = oa[:, None] + ho[:, None] * t[None, :]                     # (P, q)
    xs = sa[:, None] + hs[:, None] * t[None, :]
    po = a[eo][:, None, :] + xo[:, :, None] * (b[eo] - a[eo])[:, None, :]   # (P, q, 2)
    ps = a[es][:, None, :] + xs[:, :, None] * (b[es] - a[es])[:, None, :]
    diff = po[:, :, None, :] - ps[:, None, :, :]                     # (P, q, q, 2)
    r = np.sqrt(np.sum(diff * diff, axis=-1))
    g, hk = _hankel_pair(k, r)
    proj = -np.einsum('pijc,pc->pij', diff, normal[eo]) / np.maximum(r, G.EPS)
    dk = np.where(r > G.EPS, hk * proj, 0.0)
    P, q = len(eo), order
    ww = np.broadcast_to(np.outer(w, w).ravel(), (P, q * q))
    xo2 = np.broadcast_to(xo[:, :, None], (P, q, q)).reshape(P, q * q)
    xs2 = np.broadcast_to(xs[:, None, :], (P, q, q)).reshape(P, q * q)
    length = np.hypot(*(b - a).T)
    return _blocks(ww, g.reshape(P, -1), dk.reshape(P, -1), xo2, xs2, length[eo] * ho * length[es] * hs)


def near_all(drawn, k):
    """Every near pair's S and K' blocks of the contour, batched by rule as the reference's
    NumPy path batches them: self blocks per element (the series), touching pairs and the
    fixed 16-point pairs each in one vectorised evaluation, the close pairs refined level by
    level with every pair's unconverged boxes evaluated together.  Returns the pair count."""
    nodes, a, b, length, normal, n = _contour(drawn)
    centre = 0.5 * (a + b)
    ends = [(a[i], b[i]) for i in range(n)]
    for e in range(n):
        G.self_block(length[e], k)
    # touching pairs: element e with e - 1 (shared node: e's start) and e + 1 (e's end)
    x, y, w = G.touching_nodes()
    for obs_start in (True, False):
        eo = np.arange(n)
        es = (eo - 1) % n if obs_start else (eo + 1) % n
        d_o = (b - a) if obs_start else (a - b)
        d_s = (a - b)[es] if obs_start else (b - a)[es]
        diff = x[None, :, None] * d_o[:, None, :] - y[None, :, None] * d_s[:, None, :]
        r = np.hypot(diff[..., 0], diff[..., 1])
        g, hk = _hankel_pair(k, r)
        proj = -np.einsum('pqc,pc->pq', diff, normal[eo]) / np.maximum(r, G.EPS)
        dk = np.where(r > G.EPS, hk * proj, 0.0)
        xo = np.broadcast_to(x if obs_start else 1.0 - x, r.shape)
        xs = np.broadcast_to(1.0 - y if obs_start else y, r.shape)
        _blocks(np.broadcast_to(w, r.shape), g, dk, xo, xs, length[eo] * length[es])
    # separated near pairs
    box, close = [], []
    for e in range(n):
        ratio = np.hypot(*(centre - centre[e]).T) / np.maximum(length, length[e])
        for f in np.flatnonzero(ratio < 3.0):
            if f in (e, (e + 1) % n, (e - 1) % n):
                continue
            (close if G.needs_adaptive(ends[e], ends[f]) else box).append((e, f))
    if box:
        eo, es = np.array(box).T
        one, zero = np.ones(len(eo)), np.zeros(len(eo))
        _boxes(a, b, normal, k, eo, es, zero, one, zero, one)
    if close:
        eo, es = np.array(close).T
        floor = np.finfo(float).eps * np.maximum(1.0, length[eo] * length[es])
        one, zero = np.ones(len(eo)), np.zeros(len(eo))
        cs, ck = _boxes(a, b, normal, k, eo, es, zero, one, zero, one)
        live = [np.arange(len(eo)), zero, one, zero, one, cs, ck]
        for _depth in range(G.ADAPTIVE_MAX_DEPTH + 1):
            pid, oa, ob, sa, sb, cs, ck = live
            if not len(pid):
                break
            om, sm = 0.5 * (oa + ob), 0.5 * (sa + sb)
            kids = [(oa, om, sa, sm), (oa, om, sm, sb), (om, ob, sa, sm), (om, ob, sm, sb)]
            res = [_boxes(a, b, normal, k, eo[pid], es[pid], *kd) for kd in kids]
            fs = sum(r_[0] for r_ in res)
            fk = sum(r_[1] for r_ in res)
            ns = sum(np.linalg.norm(r_[0], axis=(1, 2)) for r_ in res)
            nk = sum(np.linalg.norm(r_[1], axis=(1, 2)) for r_ in res)
            err = np.maximum(np.linalg.norm(fs - cs, axis=(1, 2)) / np.maximum(ns, floor[pid]),
                             np.linalg.norm(fk - ck, axis=(1, 2)) / np.maximum(nk, floor[pid]))
            go = err > G.ADAPTIVE_RTOL
            live = [np.concatenate([pid[go]] * 4)] + [np.concatenate([kd[i][go] for kd in kids]) for i in range(4)] + \
                [np.concatenate([r_[0][go] for r_ in res]), np.concatenate([r_[1][go] for r_ in res])]
    return n + 2 * n + len(box) + len(close)


def far_all_compiled(drawn, k, far_block_fn, table, rows=None, order=FAR_ORDER):
    """The far pass of element rows ``rows`` (default all) through the compiled reference
    kernel."""
    nodes, a, b, length, normal, n = _contour(drawn)
    return far_rows_compiled(drawn, k, range(n) if rows is None else rows, far_block_fn, table, order)


def _loads(a, b, length, k, angles_deg, order=8):
    """Galerkin plane-wave loads of every node and angle (8 Gauss points per element, as
    ``galerkin2d.incident_loads``), vectorised over elements and angles; also returns the
    per-point phases and weights for the far field."""
    t, w = G.unit_gauss(order)
    phi = np.radians(np.asarray(angles_deg, float))
    d = np.stack([np.cos(phi), np.sin(phi)], axis=1)
    pts = a[:, None, :] + t[None, :, None] * (b - a)[:, None, :]                 # (ne, q, 2)
    phase = np.exp(1j * k * np.einsum('eqc,rc->eqr', pts, d))                    # (ne, q, R)
    wt = length[:, None] * w[None, :]
    l0 = np.einsum('eq,eqr->er', wt * (1.0 - t)[None, :], phase)
    l1 = np.einsum('eq,eqr->er', wt * t[None, :], phase)
    return l0 + np.roll(l1, 1, axis=0), phase, wt


def _far_field(x, phase, wt, normal, angles_deg, order=8):
    """Monostatic far field of the combined density x (nodes x angles), vectorised."""
    t, _w = G.unit_gauss(order)
    phi = np.radians(np.asarray(angles_deg, float))
    d = np.stack([np.cos(phi), np.sin(phi)], axis=1)
    dens = (1.0 - t)[None, :, None] * x[:, None, :] + t[None, :, None] * np.roll(x, -1, axis=0)[:, None, :]
    fac = 1.0 + normal @ d.T                                                     # (ne, R)
    return np.einsum('eq,eqr,eqr,er->r', wt, dens, phase, fac)


def time_solve(drawn, k, angles_deg, rows, far_block_fn=None, table=None, near=True):
    """Seconds of one solve: the far element-pair blocks of element rows ``rows`` (None: all;
    a sample is timed and scaled to all N rows; through the compiled reference kernel when ``far_block_fn`` is
    given, else NumPy), every near pair (``near_all``, unless ``near`` is false), then a
    LAPACK LU of an N x N complex matrix with the solve of every angle's right-hand side,
    the plane-wave loads and the far field.  Returns (seconds, parts dict)."""
    nodes, a, b, length, normal, n = _contour(drawn)
    rows = list(range(n)) if rows is None else [int(r) for r in rows]
    scale = n / max(1, len(rows))
    t_far_fill = t_near = 0.0
    if rows:
        t0 = time.perf_counter()
        if far_block_fn is not None:
            far_rows_compiled(drawn, k, rows, far_block_fn, table)
        else:
            far_rows_numpy(drawn, k, rows)
        t_far_fill = (time.perf_counter() - t0) * scale
    if near:
        t0 = time.perf_counter()
        near_all(drawn, k)
        t_near = time.perf_counter() - t0
    rng = np.random.default_rng(0)
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)) + 4.0 * np.eye(n)
    t0 = time.perf_counter()
    load, phase, wt = _loads(a, b, length, k, angles_deg)
    t_loads = time.perf_counter() - t0
    t0 = time.perf_counter()
    x = sla.lu_solve(sla.lu_factor(A, check_finite=False), -load, check_finite=False)
    t_lu = time.perf_counter() - t0
    t0 = time.perf_counter()
    _far_field(x, phase, wt, normal, angles_deg)
    t_ff = time.perf_counter() - t0
    total = t_far_fill + t_near + t_loads + t_lu + t_ff
    return total, {'far_fill_s': t_far_fill, 'near_fill_s': t_near, 'loads_s': t_loads, 'lu_solve_s': t_lu,
                   'far_field_s': t_ff, 'sampled_rows': len(rows),
                   'far_pass': 'compiled far.c' if far_block_fn is not None else 'numpy'}
