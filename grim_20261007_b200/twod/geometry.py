"""Geometry snapshot -> closed PEC contours -> straight panels (host side, FP64).

Mirrors the reference's meshing rules for the bodies this path solves (closed
perfectly conducting contours, segment TYPE 2 with IBC flag 0):

* ``twod/geometry.py:1753`` ``_build_panels``: every coordinate primitive
  (x1, y1, x2, y2) is split uniformly into a panel count given by the segment's
  ``N`` property (``_panel_count_from_n``, ``twod/geometry.py:906``): N > 0 exactly N
  panels, N < 0 |N| panels per wavelength, N = 0 the automatic
  ``DEFAULT_PANELS_PER_WAVELENGTH`` (20) per wavelength;
* ``GEOMETRY_INPUT_CHEATSHEET.md``: primitives of a segment form a head-to-tail
  chain; units "meters" or "inches";
* ``tests/general_fixtures.py:30-40``: closed contours are listed clockwise.

Other boundary kinds (impedance sheets, dielectrics, IBC) belong to formulations
outside this path and are rejected with ``NotImplementedError``.
"""
from __future__ import annotations

import itertools
import math
import operator

import numpy as np

DEFAULT_PANELS_PER_WAVELENGTH = 20
INCH = 0.0254
WELD_TOL = 1e-9


def unit_scale(units):
    u = str(units or 'inches').strip().lower()
    if u in ('m', 'meter', 'meters', 'metre', 'metres'):
        return 1.0
    if u in ('in', 'inch', 'inches'):
        return INCH
    if u in ('mm', 'millimeter', 'millimeters'):
        return 1e-3
    if u in ('cm', 'centimeter', 'centimeters'):
        return 1e-2
    raise ValueError(f'Unsupported geometry units {units!r}.')


def _flags(seg):
    props = list(seg.get('properties', []) or [])
    def geti(i, default=0):
        try:
            return int(float(props[i]))
        except (IndexError, TypeError, ValueError):
            return default
    seg_type = int(seg.get('seg_type', geti(0, 2)))
    return seg_type, geti(1, 0), geti(2, 0), geti(3, 0), geti(4, 0)


def panel_count(n_prop, length, wavelength):
    if length <= 1e-12:
        return 1
    if n_prop > 0:
        return int(n_prop)
    per = abs(n_prop) if n_prop < 0 else DEFAULT_PANELS_PER_WAVELENGTH
    if not (wavelength > 0 and math.isfinite(wavelength)):
        raise ValueError('Automatic meshing needs a positive finite wavelength.')
    return max(1, int(math.ceil(length * per / wavelength)))


_PAIR_XY = operator.itemgetter('x1', 'y1', 'x2', 'y2')


# ------------------------------------------------------------------ solver-side validation
def _window_pairs(lo, hi, tol):
    """Index pairs (i, j), i < j, whose intervals [lo, hi] overlap within tol: sort by lo,
    then for each offset d compare element p with element p + d while any window still
    reaches that far (the largest window is the few primitives stacked over one x)."""
    order = np.argsort(lo, kind='stable')
    l, h = lo[order], hi[order]
    reach = np.searchsorted(l, h + tol, side='right') - np.arange(len(l)) - 1
    pairs = []
    for d in range(1, int(reach.max(initial=0)) + 1):
        live = np.flatnonzero(reach[:len(l) - d] >= d)
        if live.size == 0:
            break
        pairs.append(np.stack([order[live], order[live + d]], axis=1))
    if not pairs:
        return np.zeros((0, 2), dtype=np.int64)
    out = np.concatenate(pairs)
    return np.sort(out, axis=1)


def _orient(px, py, qx, qy, rx, ry):
    return (qx - px) * (ry - py) - (qy - py) * (rx - px)


def validate_primitives(a, b, seg_of, prim_of, names):
    """The reference's fatal solver-side geometry checks (``twod/geometry.py:1121-1457``
    ``validate_geometry_snapshot_for_solver``) on the primitives (a -> b, metres):

    * a primitive not longer than the 1e-9 m node-weld tolerance (a degenerate element);
    * a crack: two endpoints that are not one node (farther apart than 1e-9 m) yet closer
      than the drawing tolerance min(max(1e-8, 1e-6 diagonal), half the shortest primitive
      at either), and not the two ends of one primitive;
    * two primitives with the same endpoints (a doubled boundary);
    * two primitives running along one line from a shared endpoint (collinear overlap);
    * two primitives that cross (other than neighbours of one chain).
    Raises ValueError with the reference's wording."""
    length = np.hypot(*(b - a).T)
    bad = np.flatnonzero(length <= WELD_TOL)
    if bad.size:
        i = int(bad[0])
        raise ValueError(f"Segment '{names[seg_of[i]]}' primitive {prim_of[i] + 1} is {length[i]:.3g} m long, not "
                         f"longer than the {WELD_TOL:g} m mesh node tolerance, so its two ends would be one mesh node "
                         "(a degenerate element). Remove it or merge it into a neighboring primitive.")
    pts = np.concatenate([a, b])
    span = np.ptp(pts, axis=0)
    tol = max(1e-8, 1e-6 * max(math.hypot(*span), 1.0))
    # vertices: weld endpoints within 1e-9 m into nodes
    key = np.round(pts / WELD_TOL).astype(np.int64)
    # node of each endpoint: rows of key numbered in lexicographic order (np.unique(axis=0)
    # numbers them the same way but sorts the rows as bytes, ten times slower)
    order = np.lexsort((key[:, 1], key[:, 0]))
    ks = key[order]
    first_of_run = np.ones(len(ks), dtype=bool)
    first_of_run[1:] = np.any(ks[1:] != ks[:-1], axis=1)
    node = np.empty(len(ks), dtype=np.int64)
    node[order] = np.cumsum(first_of_run) - 1
    nprim = len(a)
    feature = np.full(int(node.max()) + 1, np.inf)
    np.minimum.at(feature, node, np.concatenate([length, length]))
    vpt = np.zeros((len(feature), 2))
    vpt[node] = pts
    # cracks
    vp = _window_pairs(vpt[:, 0], vpt[:, 0], tol)
    if len(vp):
        gap = np.hypot(*(vpt[vp[:, 0]] - vpt[vp[:, 1]]).T)
        local = np.minimum(tol, 0.5 * np.minimum(feature[vp[:, 0]], feature[vp[:, 1]]))
        ends = np.sort(np.stack([node[:nprim], node[nprim:]], axis=1), axis=1)
        nv = np.int64(len(feature))
        is_end = np.isin(vp[:, 0] * nv + vp[:, 1], ends[:, 0] * nv + ends[:, 1])
        crack = np.flatnonzero((gap > WELD_TOL) & (gap <= local) & ~is_end)
        if crack.size:
            i, j = vp[crack[0]]
            g = gap[crack[0]]
            (px, py), (qx, qy) = vpt[i], vpt[j]
            raise ValueError(f"Geometry crack: endpoints ({px:.9g}, {py:.9g}) m and ({qx:.9g}, {qy:.9g}) m are "
                             f"{g:.3g} m apart -- close enough to look connected, but beyond the 1e-9 m mesh "
                             "node-snap tolerance, so they would mesh as an OPEN gap. Make the endpoints exactly "
                             "coincident (or separate them intentionally).")
    # primitive pairs with overlapping bounding boxes
    xlo, xhi = np.minimum(a[:, 0], b[:, 0]), np.maximum(a[:, 0], b[:, 0])
    ylo, yhi = np.minimum(a[:, 1], b[:, 1]), np.maximum(a[:, 1], b[:, 1])
    pp = _window_pairs(xlo, xhi, tol)
    if not len(pp):
        return
    i, j = pp[:, 0], pp[:, 1]
    keep = (ylo[j] <= yhi[i] + tol) & (ylo[i] <= yhi[j] + tol)
    i, j = i[keep], j[keep]
    feat = np.minimum(length, np.minimum(feature[node[:nprim]], feature[node[nprim:]]))
    ptol = np.minimum(tol, 0.5 * np.minimum(feat[i], feat[j]))
    a1, a2, b1, b2 = a[i], b[i], a[j], b[j]
    close = lambda p, q, t: np.hypot(*(p - q).T) <= t
    dup = (close(a1, b1, ptol) & close(a2, b2, ptol)) | (close(a1, b2, ptol) & close(a2, b1, ptol))
    if dup.any():
        q = int(np.flatnonzero(dup)[0])
        raise ValueError(f"Duplicate primitive: '{names[seg_of[i[q]]]}' primitive {prim_of[i[q]] + 1} and "
                         f"'{names[seg_of[j[q]]]}' primitive {prim_of[j[q]] + 1} have identical endpoints. Remove "
                         "one -- a doubled boundary doubles the surface currents.")
    na1, na2, nb1, nb2 = node[i], node[nprim + i], node[j], node[nprim + j]
    share = (na1 == nb1) | (na1 == nb2) | (na2 == nb1) | (na2 == nb2)
    # from the shared endpoint: u along primitive i, v along primitive j
    a_first = (na1 == nb1) | (na1 == nb2)
    b_first = (nb1 == na1) | (nb1 == na2)
    u = np.where(a_first[:, None], a2 - a1, a1 - a2)
    v = np.where(b_first[:, None], b2 - b1, b1 - b2)
    lu, lv = np.hypot(*u.T), np.hypot(*v.T)
    den = np.maximum(lu * lv, 1e-300)
    along = share & (lu > 1e-12) & (lv > 1e-12) & (np.abs(u[:, 0] * v[:, 1] - u[:, 1] * v[:, 0]) / den < 1e-7) & \
        (np.sum(u * v, axis=1) / den > 0.0) & (np.minimum(lu, lv) > WELD_TOL)
    if along.any():
        q = int(np.flatnonzero(along)[0])
        raise ValueError(f"Collinear overlapping primitives: '{names[seg_of[i[q]]]}' primitive {prim_of[i[q]] + 1} "
                         f"and '{names[seg_of[j[q]]]}' primitive {prim_of[j[q]] + 1} run along the same line from a "
                         f"shared endpoint, overlapping for {min(lu[q], lv[q]):.3g} m. Split or remove the overlapping "
                         "span.")
    rest = ~share & ~((seg_of[i] == seg_of[j]) & (np.abs(prim_of[i] - prim_of[j]) <= 1))
    i, j, ptol = i[rest], j[rest], ptol[rest]
    a1, a2, b1, b2 = a[i], b[i], a[j], b[j]
    endclose = close(a1, b1, ptol) | close(a1, b2, ptol) | close(a2, b1, ptol) | close(a2, b2, ptol)
    o1 = _orient(*a1.T, *a2.T, *b1.T)
    o2 = _orient(*a1.T, *a2.T, *b2.T)
    o3 = _orient(*b1.T, *b2.T, *a1.T)
    o4 = _orient(*b1.T, *b2.T, *a2.T)
    ta = ptol * np.maximum(np.hypot(*(a2 - a1).T), 1e-12)
    tb = ptol * np.maximum(np.hypot(*(b2 - b1).T), 1e-12)

    def on_seg(p, q, r):
        return ((np.minimum(p[:, 0], r[:, 0]) - ptol <= q[:, 0]) & (q[:, 0] <= np.maximum(p[:, 0], r[:, 0]) + ptol) &
                (np.minimum(p[:, 1], r[:, 1]) - ptol <= q[:, 1]) & (q[:, 1] <= np.maximum(p[:, 1], r[:, 1]) + ptol))
    cross = (((o1 > ta) & (o2 < -ta)) | ((o1 < -ta) & (o2 > ta))) & (((o3 > tb) & (o4 < -tb)) | ((o3 < -tb) & (o4 > tb)))
    touch = ((np.abs(o1) <= ta) & on_seg(a1, b1, a2)) | ((np.abs(o2) <= ta) & on_seg(a1, b2, a2)) | \
        ((np.abs(o3) <= tb) & on_seg(b1, a1, b2)) | ((np.abs(o4) <= tb) & on_seg(b1, a2, b2))
    hit = ~endclose & (cross | touch)
    if hit.any():
        q = int(np.flatnonzero(hit)[0])
        raise ValueError(f"Geometry contains an unsupported segment intersection between '{names[seg_of[i[q]]]}' "
                         f"primitive {prim_of[i[q]] + 1} and '{names[seg_of[j[q]]]}' primitive {prim_of[j[q]] + 1}.")


def validate_winding(polygons, names):
    """The reference's winding rule for closed PEC contours (``geometry/io.py:712``
    ``check_orientation_consistency``): a contour enclosed by an even number of others must
    run clockwise (its normals into the unbounded air), one enclosed by an odd number
    counter-clockwise (a void)."""
    areas = [0.5 * float(np.sum(v[:, 0] * np.roll(v[:, 1], -1) - np.roll(v[:, 0], -1) * v[:, 1])) for v in polygons]
    for idx, v in enumerate(polygons):
        depth = 0
        x, y = v[0]
        for jdx, w in enumerate(polygons):
            if jdx == idx:
                continue
            xa, ya, xb, yb = w[:, 0], w[:, 1], np.roll(w[:, 0], -1), np.roll(w[:, 1], -1)
            crosses = ((ya > y) != (yb > y)) & (x < xa + (y - ya) * (xb - xa) / np.where(yb != ya, yb - ya, 1.0))
            depth += int(np.count_nonzero(crosses) % 2)
        want_cw = depth % 2 == 0
        if (areas[idx] < 0.0) != want_cw:
            raise ValueError("Geometry orientation check failed:\n  - "
                             f"segment '{names[idx]}' is a closed PEC contour at nesting depth {depth}; it must run "
                             f"{'clockwise' if want_cw else 'counter-clockwise'} so that its normals point into the air.")


def contours_from_snapshot(snapshot, geometry_units='inches', wavelength=None, max_panels=20000, checks=None):
    """Return a list of closed polygons (vertex arrays, metres) ready for ``panel_geometry``,
    after the reference's fatal geometry checks (``validate_primitives``, ``validate_winding``).
    With a list ``checks`` those two checks are not run here: a callable that runs them (and
    raises their ValueError) is appended instead, for the caller to run alongside the solve
    and before it returns anything."""
    scale = unit_scale(geometry_units)
    segs = list(snapshot.get('segments', []) or [])
    if not segs:
        raise ValueError('Geometry snapshot has no segments.')
    if snapshot.get('dielectrics') or snapshot.get('ibcs'):
        raise NotImplementedError('Dielectric and impedance boundaries are outside the GPU PEC solve path.')
    polygons = []
    total = 0
    prim_a, prim_b, seg_of, prim_of, names, poly_names = [], [], [], [], [], []
    for seg in segs:
        seg_type, n_prop, ibc, pos, neg = _flags(seg)
        if seg_type != 2 or ibc != 0 or pos != 0 or neg != 0:
            raise NotImplementedError(
                f"Segment {seg.get('name', '?')!r}: only closed PEC contours (TYPE 2, IBC 0) are solved on the GPU path.")
        pairs = seg.get('point_pairs', []) or []
        if not pairs:
            continue
        xy = np.fromiter(itertools.chain.from_iterable(map(_PAIR_XY, pairs)), np.float64,
                         4 * len(pairs)).reshape(-1, 4) * scale
        a, b = xy[:, :2], xy[:, 2:]
        prim_a.append(a)
        prim_b.append(b)
        seg_of.append(np.full(len(a), len(names)))
        prim_of.append(np.arange(len(a)))
        names.append(str(seg.get('name', f'segment_{len(names) + 1}')))
        lengths = np.hypot(b[:, 0] - a[:, 0], b[:, 1] - a[:, 1])
        if n_prop > 0:
            cnt = np.full(len(pairs), int(n_prop), dtype=np.int64)
        else:
            cnt = np.array([panel_count(n_prop, float(L), wavelength) for L in lengths], dtype=np.int64)
        gaps = np.hypot(*(b[:-1] - a[1:]).T)
        tol = np.maximum(WELD_TOL, 1e-9 * np.maximum(1.0, lengths[1:]))
        if np.any(gaps > tol):
            k = int(np.flatnonzero(gaps > tol)[0]) + 1
            raise ValueError(f"Segment '{names[-1]}' has a disconnected primitive chain between elements {k} and "
                             f"{k + 1}. Primitives within one segment must chain head-to-tail; put disconnected "
                             "geometry in separate segments.")
        # panel vertices a + i (b - a) / cnt, i < cnt, of every primitive (linspace's i * (1 / cnt))
        owner = np.repeat(np.arange(len(pairs)), cnt)
        first = np.cumsum(cnt) - cnt
        step = 1.0 / cnt.astype(np.float64)
        t = (np.arange(int(cnt.sum())) - first[owner]) * step[owner]
        poly = a[owner] + t[:, None] * (b - a)[owner]
        pts_last = b[-1]
        if np.hypot(*(pts_last - poly[0])) > max(WELD_TOL, 1e-9):
            raise ValueError(f"Segment {seg.get('name', '?')!r} is not closed; open contours are outside this path.")
        total += len(poly)
        if total > int(max_panels):
            raise ValueError('Discretization exceeds the configured panel limit.')
        polygons.append(poly)
        poly_names.append(names[-1])
    if prim_a:
        args = (np.concatenate(prim_a), np.concatenate(prim_b), np.concatenate(seg_of), np.concatenate(prim_of), names)

        def check(args=args, polygons=list(polygons), poly_names=list(poly_names)):
            validate_primitives(*args)
            validate_winding(polygons, poly_names)
        if checks is None:
            check()
        else:
            checks.append(check)
    return polygons


def panel_geometry(polygons):
    """Polygons -> (n, 7) FP64 array of (cx, cy, tx, ty, h, nx, ny), outward normals."""
    rows = []
    for v in polygons:
        v = np.asarray(v, dtype=np.float64)
        b = np.roll(v, -1, axis=0)
        area = 0.5 * np.sum(v[:, 0] * b[:, 1] - b[:, 0] * v[:, 1])
        edge = b - v
        length = np.hypot(edge[:, 0], edge[:, 1])
        if np.any(length <= 0):
            raise ValueError('Zero-length panel.')
        t = edge / length[:, None]
        s = 1.0 if area < 0.0 else -1.0
        nrm = s * np.stack([-t[:, 1], t[:, 0]], axis=1)
        c = 0.5 * (v + b)
        rows.append(np.column_stack([c, t, 0.5 * length, nrm]))
    return np.ascontiguousarray(np.concatenate(rows, axis=0))


def te_curvature_correction(polygons):
    """Per-panel TE diagonal correction (kappa_start + kappa_end)/2 * L / (4 pi).

    The straight self panel drops the smooth-curve diagonal limit kappa/(4 pi) of the
    normal-derivative kernel; the curvature at each vertex is the turning angle over
    the mean adjacent panel length (convex turns positive), and vertices turning by
    more than 20 degrees are true corners (kappa = 0).
    """
    out = []
    corner = math.radians(20.0)
    for v in polygons:
        v = np.asarray(v, dtype=np.float64)
        b = np.roll(v, -1, axis=0)
        area = 0.5 * np.sum(v[:, 0] * b[:, 1] - b[:, 0] * v[:, 1])
        o = 1.0 if area > 0.0 else -1.0
        edge = b - v
        length = np.hypot(edge[:, 0], edge[:, 1])
        t = edge / length[:, None]
        tp = np.roll(t, 1, axis=0)
        lp = np.roll(length, 1)
        cross = tp[:, 0] * t[:, 1] - tp[:, 1] * t[:, 0]
        dot = tp[:, 0] * t[:, 0] + tp[:, 1] * t[:, 1]
        beta = o * np.arctan2(cross, dot)
        kappa = np.where(np.abs(beta) <= corner, beta / (0.5 * (lp + length)), 0.0)
        out.append(0.5 * (kappa + np.roll(kappa, -1)) * length / (4.0 * math.pi))
    return np.ascontiguousarray(np.concatenate(out))


def perimeter(polygons):
    return float(sum(np.sum(np.hypot(*(np.roll(v, -1, axis=0) - v).T)) for v in polygons))
