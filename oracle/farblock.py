"""CPU restatement of the reference's far-field Galerkin block quadrature (TEST INFRASTRUCTURE).

Only the tests import this module: it is the checker of the GPU far-block kernel, never a
product path.  It restates ``twod/assembly/native/far.c:26-186`` (``asymptotic``,
``kernel``, ``first_or_add``, ``ghost_far_block_impl``) in plain Python floats, operation
for operation and in the same order (Python floats round every operation on its own, as
the reference's ``-ffp-contract=off`` build does), so pairs inside the kernel table
reproduce the reference bit for bit; beyond the table the complex exponential and square
root are Python's ``cmath`` (agreement to a few ulp).  Pure-Python loops: small cases only.

Pinned against the reference's own compiled kernel through ``tests/golden/far_block.npz``
(made by ``tests/golden/make_far_golden.py``).
"""
from __future__ import annotations

import cmath
import math

import numpy as np

EPS = 1e-12


def asymptotic(k, r):
    """(j/4) H0^(2)(kr) and (j/4) k H1^(2)(kr), 8-term large-argument expansion (far.c:26-46)."""
    z = k * r
    root = cmath.sqrt(2.0 / (math.pi * z))
    out = []
    for nu in range(2):
        mu = 4.0 * nu * nu
        term, total, factor = 1.0 + 0j, 1.0 + 0j, -1j / z
        for m in range(1, 8):
            odd = 2.0 * m - 1.0
            term *= (mu - odd * odd) / (8.0 * m) * factor
            total += term
        phase = cmath.exp(-1j * (z - nu * math.pi / 2.0 - math.pi / 4.0))
        value = 0.25j * root * phase * total
        if nu == 1:
            value *= k
        out += [value.real, value.imag]
    return out


def kernel(k, bounds, coeff, degree, r):
    """Kernel values at r, or None below the table (far.c:49-83).  coeff: flat doubles,
    [interval][power][channel][re, im]."""
    intervals = len(bounds) - 1
    if not (r >= bounds[0]):
        return None
    if r > bounds[intervals]:
        return asymptotic(k, r)
    lo, hi = 0, intervals
    while lo + 1 < hi:
        mid = lo + (hi - lo) // 2
        if r < bounds[mid]:
            hi = mid
        else:
            lo = mid
    x = (r - bounds[lo]) / (bounds[lo + 1] - bounds[lo])
    base = lo * (degree + 1) * 4
    out = []
    for c in range(2):
        off = 2 * c
        re = coeff[base + 4 * degree + off]
        im = coeff[base + 4 * degree + off + 1]
        for j in range(degree - 1, -1, -1):
            re = re * x + coeff[base + 4 * j + off]
            im = im * x + coeff[base + 4 * j + off + 1]
        out += [re, im]
    return out


def far_block(obs_pts, src_pts, qw, phi, obs_norm, src_norm, far, obs_normal_deriv, want_s, want_k, mirrored, k,
              bounds, coeff):
    """Accumulators (width^2, mb, nb) complex128 for S, K and mirrored K from zero, or None
    when a far distance falls below the table (the reference's status 2)."""
    obs_pts = np.asarray(obs_pts, float)
    src_pts = np.asarray(src_pts, float)
    mb, q = obs_pts.shape[:2]
    nb = src_pts.shape[0]
    width = np.asarray(phi).shape[1]
    coeff = np.ascontiguousarray(coeff).view(np.float64).ravel().tolist()
    degree = len(coeff) // (4 * (len(bounds) - 1)) - 1
    bounds = [float(b) for b in bounds]
    qw = [float(w) for w in qw]
    phi = np.asarray(phi, float).tolist()
    k = complex(k)
    with_kt = want_k and mirrored
    shape = (width * width, mb, nb)
    acc_s = np.zeros(shape, complex) if want_s else None
    acc_k = np.zeros(shape, complex) if want_k else None
    acc_kt = np.zeros(shape, complex) if with_kt else None
    for i in range(mb):
        on = [float(v) for v in obs_norm[i]]
        for j in range(nb):
            if not far[i][j]:
                continue
            sn = [float(v) for v in src_norm[j]]
            n_ij = on if obs_normal_deriv else sn
            n_ji = sn if obs_normal_deriv else on
            a_s = [[0.0, 0.0] for _ in range(width * width)]
            a_k = [[0.0, 0.0] for _ in range(width * width)]
            a_kt = [[0.0, 0.0] for _ in range(width * width)]
            for qi in range(q):
                ps = [[0.0, 0.0] for _ in range(width)]
                pk = [[0.0, 0.0] for _ in range(width)]
                pkt = [[0.0, 0.0] for _ in range(width)]
                ox, oy = float(obs_pts[i, qi, 0]), float(obs_pts[i, qi, 1])
                for qj in range(q):
                    dx = ox - float(src_pts[j, qj, 0])
                    dy = oy - float(src_pts[j, qj, 1])
                    dist = math.sqrt(dx * dx + dy * dy)
                    if not (dist >= EPS):
                        dist = EPS
                    value = kernel(k, bounds, coeff, degree, dist)
                    if value is None:
                        return None
                    w = qw[qj]
                    first = qj == 0
                    dk_re = dk_im = 0.0
                    if want_k:
                        proj = dx * n_ij[0] + dy * n_ij[1]
                        proj = proj / dist
                        dk_re, dk_im = value[2] * proj, value[3] * proj
                        if obs_normal_deriv:
                            dk_re, dk_im = -dk_re, -dk_im
                    for b in range(width):
                        c = w * phi[qj][b]
                        if want_s:
                            _first_or_add(ps[b], first, value[0], value[1], c)
                        if want_k:
                            _first_or_add(pk[b], first, dk_re, dk_im, c)
                    if with_kt:
                        proj = dx * n_ji[0] + dy * n_ji[1]
                        proj = proj / dist
                        re, im = value[2] * proj, value[3] * proj
                        if not obs_normal_deriv:
                            re, im = -re, -im
                        for a in range(width):
                            _first_or_add(pkt[a], first, re, im, w * phi[qj][a])
                wo = qw[qi]
                for a in range(width):
                    c = wo * phi[qi][a]
                    for b in range(width):
                        ab = width * a + b
                        if want_s:
                            a_s[ab] = [a_s[ab][0] + ps[b][0] * c, a_s[ab][1] + ps[b][1] * c]
                        if want_k:
                            a_k[ab] = [a_k[ab][0] + pk[b][0] * c, a_k[ab][1] + pk[b][1] * c]
                if with_kt:
                    for b in range(width):
                        c = wo * phi[qi][b]
                        for a in range(width):
                            ab = width * a + b
                            a_kt[ab] = [a_kt[ab][0] + pkt[a][0] * c, a_kt[ab][1] + pkt[a][1] * c]
            for ab in range(width * width):
                if want_s:
                    acc_s[ab, i, j] = complex(*a_s[ab])
                if want_k:
                    acc_k[ab, i, j] = complex(*a_k[ab])
                if with_kt:
                    acc_kt[ab, i, j] = complex(*a_kt[ab])
    return acc_s, acc_k, acc_kt


def _first_or_add(acc, first, re, im, c):
    if first:
        acc[0], acc[1] = re * c, im * c
    else:
        acc[0], acc[1] = acc[0] + re * c, acc[1] + im * c


def in_table(obs_pts, src_pts, far, upper):
    """(mb, nb) mask of far pairs whose every quadrature distance lies inside the table."""
    d = np.sqrt(((np.asarray(obs_pts)[:, None, :, None, :] - np.asarray(src_pts)[None, :, None, :, :]) ** 2).sum(-1))
    return np.asarray(far, bool) & (d.max(axis=(2, 3)) <= upper)
