"""Element-pair routing and near-pair point rules of the body-of-revolution fill.

The reference integrates an element pair one of three ways (``bor/solver.py:1509-1580``
``_configure_near_pair_routing``, ``:795`` ``_same_surface_points``, ``:843``
``_regular_cell_points``); the GPU kernels take the same routing and point sets:

* class 1 -- self and adjacent pairs: graded cells.  The unit square (s on the test
  element, s' on the source element) is split recursively, to depth 4, toward the
  singular set (the diagonal s = s' for a self pair, the shared corner for an adjacent
  pair), every cell carrying a tensor rule of 4 (in s) x 5 (in s') Gauss points
  (``bor/solver.py:718-792`` ``_graded_cells`` / ``_cell_points``);
* class 2 -- every other pair with |e - f| <= 2, and any pair whose segments come within
  max(1.001 * 8 * 2 pi / 8192 * rho_max(e, f), 2 max(L_e, L_f)): a 12 x 12 Gauss tensor rule;
* class 0 -- the rest: 3 x 3 Gauss points (``bor/kernels.py:41`` ``FAR_GAUSS_ORDER``).
"""
from __future__ import annotations

import math

import numpy as np

FAR_ORDER = 3
CELL_ORDER = 4
CELL_DEPTH = 4
REGULAR_ORDER = 12
NEAR_SPAN = 2
DIRECT_SCALE = 1.001 * 8.0 * 2.0 * math.pi / 8192


def _unit_gauss(q):
    x, w = np.polynomial.legendre.leggauss(q)
    return 0.5 * (x + 1.0), 0.5 * w


def _segment_distance(c, a, b):
    """Distance from points c to segments [a, b] (arrays [..., 2], broadcast)."""
    ab = b - a
    t = np.sum((c - a) * ab, axis=-1) / np.maximum(np.sum(ab * ab, axis=-1), 1e-300)
    d = c - (a + np.clip(t, 0.0, 1.0)[..., None] * ab)
    return np.hypot(d[..., 0], d[..., 1])


def pair_classes(nodes):
    """(ne, ne) uint8 routing of every element pair: 0 far, 1 self / adjacent, 2 other near."""
    nodes = np.asarray(nodes, dtype=np.float64)
    ne = len(nodes) - 1
    a, b = nodes[:-1], nodes[1:]
    lengths = np.hypot(*(b - a).T)
    rho_e = np.maximum(a[:, 0], b[:, 0])
    idx = np.arange(ne)
    apart = np.abs(idx[:, None] - idx[None, :])
    cls = np.zeros((ne, ne), dtype=np.uint8)
    cls[apart <= NEAR_SPAN] = 2
    cls[apart <= 1] = 1
    # candidates by the centre-distance lower bound (the reference's prefilter), then the
    # exact segment distance
    mids = 0.5 * (a + b)
    half = 0.5 * lengths
    d = np.hypot(mids[:, None, 0] - mids[None, :, 0], mids[:, None, 1] - mids[None, :, 1])
    gap = np.maximum(DIRECT_SCALE * np.maximum(rho_e[:, None], rho_e[None, :]),
                     2.0 * np.maximum(lengths[:, None], lengths[None, :]))
    cand = np.nonzero((apart > NEAR_SPAN) & (d - half[:, None] - half[None, :] <= gap))
    if len(cand[0]):
        e, f = cand
        dist = np.minimum(np.minimum(_segment_distance(a[e], a[f], b[f]), _segment_distance(b[e], a[f], b[f])),
                          np.minimum(_segment_distance(a[f], a[e], b[e]), _segment_distance(b[f], a[e], b[e])))
        near = dist <= gap[e, f]
        cls[e[near], f[near]] = 2
    return cls


def _graded_cells(kind, depth):
    """Cells (s0, s1, p0, p1) of the unit square refined toward 'diag' (s = s') or the
    corner 'cornerAB' (s = A, s' = B)."""
    cells = []
    stack = [(0.0, 1.0, 0.0, 1.0, 0)]
    while stack:
        s0, s1, p0, p1, d = stack.pop()
        if kind == 'diag':
            touches = not (s1 <= p0 or p1 <= s0)
        else:
            ca, cb = float(kind[6]), float(kind[7])
            touches = s0 <= ca <= s1 and p0 <= cb <= p1
        if d >= depth or not touches:
            cells.append((s0, s1, p0, p1))
            continue
        sm, pm = 0.5 * (s0 + s1), 0.5 * (p0 + p1)
        # pushed in reverse so that cells come out in the recursive order
        stack += [(sm, s1, pm, p1, d + 1), (sm, s1, p0, pm, d + 1), (s0, sm, pm, p1, d + 1), (s0, sm, p0, pm, d + 1)]
    return cells


def _cell_rule(kind):
    u, wu = _unit_gauss(CELL_ORDER)
    v, wv = _unit_gauss(CELL_ORDER + 1)
    out = []
    for s0, s1, p0, p1 in _graded_cells(kind, CELL_DEPTH):
        hs, hp = s1 - s0, p1 - p0
        a, b = np.meshgrid(s0 + u * hs, p0 + v * hp, indexing='ij')
        out.append(np.stack([a.ravel(), b.ravel(), np.outer(wu * hs, wv * hp).ravel()], axis=1))
    return np.concatenate(out)


def near_rules():
    """(rule [n, 3] of (s, s', w), starts [5]): the self, adjacent f = e + 1, adjacent
    f = e - 1 and regular near point sets, concatenated."""
    u, w = _unit_gauss(REGULAR_ORDER)
    a, b = np.meshgrid(u, u, indexing='ij')
    regular = np.stack([a.ravel(), b.ravel(), np.outer(w, w).ravel()], axis=1)
    parts = [_cell_rule('diag'), _cell_rule('corner10'), _cell_rule('corner01'), regular]
    starts = np.cumsum([0] + [len(p) for p in parts]).astype(np.int32)
    return np.ascontiguousarray(np.concatenate(parts)), starts
