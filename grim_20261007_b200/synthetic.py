"""Seeded synthetic geometries for the benchmark and test workloads.

Every generator returns plain NumPy arrays:

* 2-D bodies: a closed polygon, vertices (N, 2) in metres, listed CLOCKWISE
  without repeating the first vertex (the reference requires clockwise contours,
  ``ghost_backend/tests/general_fixtures.py:30-40`` reverses counter-clockwise ones);
  ``snapshot_from_polygons`` turns polygons into the reference's geometry snapshot
  dict (``twod/geometry.py:1121`` ``prepare_geometry`` input: segments with
  ``seg_type``, five string ``properties`` and ``point_pairs``).
* Bodies of revolution: a generatrix (N+1, 2) of (rho, z) nodes from the +z pole to
  the -z pole (``bor/solver.py:3337`` ``_validate_solve_bor_generatrix``).
"""
from __future__ import annotations

import math

import numpy as np

C0 = 299_792_458.0


def circle(radius, n):
    """Regular n-gon inscribed in a circle, vertex 0 at (radius, 0), clockwise."""
    th = -2.0 * np.pi * np.arange(n) / n
    return np.stack([radius * np.cos(th), radius * np.sin(th)], axis=1)


def naca_symmetric(thickness, n, chord=1.0, closed_te=False):
    """NACA 00tt airfoil with cosine node spacing, ``n`` elements in total (even), clockwise.

    Half-thickness y_t = 5 t c [0.2969 sqrt(x) - 0.1260 x - 0.3516 x^2 + 0.2843 x^3 + a4 x^4].

    * default: the standard a4 = -0.1015.  The trailing edge keeps a finite thickness
      2 y_t(c) = 0.021 t c; its base is closed by two straight elements through (c, 0), and
      each surface has n/2 - 1 elements.  Vertices start at (c, 0), go down the base, along
      the lower surface to the leading edge and back along the upper surface.
    * ``closed_te``: a4 = -0.1036, y_t(c) = 0, a sharp trailing edge and n/2 elements per
      surface, starting at the trailing edge.  At high element counts the upper and lower
      vertices next to its tip come closer (7e-7 m at n = 2048, t = 12 %) than the
      reference's crack tolerance, and the reference refuses the contour.
    """
    if n % 2:
        raise ValueError("NACA panel count must be even")
    a4 = -0.1036 if closed_te else -0.1015
    m = n // 2 if closed_te else n // 2 - 1
    if m < 2:
        raise ValueError("NACA panel count too small")
    beta = np.pi * np.arange(m + 1) / m
    x = 0.5 * (1.0 + np.cos(beta))  # 1 -> 0
    yt = 5.0 * thickness * (0.2969 * np.sqrt(x) - 0.1260 * x - 0.3516 * x ** 2 + 0.2843 * x ** 3 + a4 * x ** 4)
    yt[-1] = 0.0
    if closed_te:
        yt[0] = 0.0
    lower = np.stack([x * chord, -yt * chord], axis=1)            # TE -> LE along the lower surface
    upper = np.stack([x[::-1] * chord, yt[::-1] * chord], axis=1)  # LE -> TE along the upper surface
    if closed_te:
        return np.concatenate([lower[:-1], upper[:-1]], axis=0)
    return np.concatenate([[[chord, 0.0]], lower, upper[1:]], axis=0)


def superellipse(a, b, p, n):
    """|x/a|^p + |y/b|^p = 1 sampled uniformly in the parameter, clockwise."""
    t = -2.0 * np.pi * np.arange(n) / n
    c, s = np.cos(t), np.sin(t)
    x = a * np.sign(c) * np.abs(c) ** (2.0 / p)
    y = b * np.sign(s) * np.abs(s) ** (2.0 / p)
    return np.stack([x, y], axis=1)


def polygon_perimeter(verts):
    d = np.roll(verts, -1, axis=0) - verts
    return float(np.sum(np.hypot(d[:, 0], d[:, 1])))


def airfoil_case(seed, n=2048, panels_per_wavelength=10.0, chord=1.0):
    """Seeded NACA 00tt (tt ~ U[8, 15] %) with N panels at lambda/``panels_per_wavelength``.

    Returns (vertices, k, frequency_hz, thickness).
    """
    rng = np.random.default_rng(seed)
    t = float(rng.uniform(0.08, 0.15))
    v = naca_symmetric(t, n, chord)
    lam = polygon_perimeter(v) * panels_per_wavelength / n
    k = 2.0 * math.pi / lam
    return v, k, C0 / lam, t


def airfoil_sweep_case(seed, nfreq=256, band=20.0, nmin=64, nmax=4096, panels_per_wavelength=10.0, chord=1.0):
    """Seeded NACA 00tt frequency sweep: ``nfreq`` frequencies log-spaced over ``band``:1
    up to the frequency where lambda / ``panels_per_wavelength`` panels give ``nmax``; at
    each, N = perimeter * ppw / lambda rounded to even, clipped to [nmin, nmax], cosine-spaced
    panels.

    Returns ([(vertices, k, frequency_hz), ...], thickness).
    """
    rng = np.random.default_rng(seed)
    t = float(rng.uniform(0.08, 0.15))
    perimeter = polygon_perimeter(naca_symmetric(t, 8192, chord))
    f_max = C0 * nmax / (perimeter * panels_per_wavelength)
    cases = []
    for f in np.geomspace(f_max / band, f_max, nfreq):
        lam = C0 / f
        n = int(min(nmax, max(nmin, 2 * round(0.5 * perimeter * panels_per_wavelength / lam))))  # even
        cases.append((naca_symmetric(t, n, chord), 2.0 * math.pi / lam, float(f)))
    return cases, t


def snapshot_from_polygons(polygons, name='body'):
    """Reference geometry snapshot: one PEC segment (TYPE 2, N=1) per closed polygon."""
    segments = []
    for i, v in enumerate(polygons):
        v = np.asarray(v, dtype=np.float64)
        w = np.roll(v, -1, axis=0)
        pairs = [dict(x1=float(a[0]), y1=float(a[1]), x2=float(b[0]), y2=float(b[1])) for a, b in zip(v, w)]
        segments.append(dict(name=f'{name}{i}', seg_type=2, properties=['2', '1', '0', '0', '0'],
                             point_pairs=pairs))
    return dict(segments=segments, ibcs=[], dielectrics=[])


def sphere_generatrix(radius, n):
    t = np.linspace(0.0, np.pi, n + 1)
    pts = np.stack([radius * np.sin(t), radius * np.cos(t)], axis=1)
    pts[0, 0] = 0.0
    pts[-1, 0] = 0.0
    return pts


def ogive_generatrix(length, half_angle_deg, n):
    """Closed double ogive: a circular arc of half-angle alpha at the tips rotated about z.

    R = (L/2)/sin(alpha), rho(z) = sqrt(R^2 - z^2) - R cos(alpha), tips at z = +-L/2.
    Nodes uniform in arc angle, from the +z tip to the -z tip.
    """
    alpha = math.radians(half_angle_deg)
    r_arc = 0.5 * length / math.sin(alpha)
    ang = np.linspace(alpha, -alpha, n + 1)  # polar angle of the arc point seen from the arc centre
    z = r_arc * np.sin(ang)
    rho = r_arc * np.cos(ang) - r_arc * math.cos(alpha)
    rho[0] = 0.0
    rho[-1] = 0.0
    return np.stack([np.maximum(rho, 0.0), z], axis=1)


def ogive_case(seed, n=400):
    rng = np.random.default_rng(seed)
    length = float(rng.uniform(2.0, 4.0))
    half = float(rng.uniform(15.0, 30.0))
    return ogive_generatrix(length, half, n), length, half
