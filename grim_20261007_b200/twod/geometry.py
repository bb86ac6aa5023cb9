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


def contours_from_snapshot(snapshot, geometry_units='inches', wavelength=None, max_panels=20000):
    """Return a list of closed polygons (vertex arrays, metres) ready for ``panel_geometry``."""
    scale = unit_scale(geometry_units)
    segs = list(snapshot.get('segments', []) or [])
    if not segs:
        raise ValueError('Geometry snapshot has no segments.')
    if snapshot.get('dielectrics') or snapshot.get('ibcs'):
        raise NotImplementedError('Dielectric and impedance boundaries are outside the GPU PEC solve path.')
    polygons = []
    total = 0
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
        lengths = np.hypot(b[:, 0] - a[:, 0], b[:, 1] - a[:, 1])
        if n_prop > 0:
            cnt = np.full(len(pairs), int(n_prop), dtype=np.int64)
        else:
            cnt = np.array([panel_count(n_prop, float(L), wavelength) for L in lengths], dtype=np.int64)
        gaps = np.hypot(*(b[:-1] - a[1:]).T)
        tol = np.maximum(WELD_TOL, 1e-9 * np.maximum(1.0, lengths[1:]))
        if np.any(gaps > tol):
            raise ValueError(f"Segment {seg.get('name', '?')!r}: primitives do not form a head-to-tail chain.")
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
