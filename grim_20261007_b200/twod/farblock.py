"""Far-field Galerkin element-pair blocks on the GPU, behind the reference's native interface.

``far_block`` has the arguments, result and fallback contract of the reference's
``twod/assembly/native/far.py:201-249`` ``far_block``: accumulators (width^2, mb, nb)
complex128 for S, K and the mirrored K of the far pairs (zero elsewhere), or None when a
far distance falls below the kernel table (the caller then takes its NumPy path).  The
work runs in ``ghost_far_block`` of libgrimgpu (``include/grimgpu.h``), which has the exact
C signature of the reference's ``far.c:193`` export, so the reference can also load the
library directly in place of its ``libghost_far.so``.  Results inside the table equal the
reference's bit for bit (same operations in the same order, no fused multiply-add).
"""
from __future__ import annotations

import numpy as np

from .. import _lib


def _double(value):
    return np.ascontiguousarray(value, dtype=np.float64)


def far_block(table, k, obs_pts, src_pts, weights, phi, obs_normals, src_normals, far, obs_normal_deriv, want_s,
              want_k, mirrored):
    """GPU ``far_block``; ``table`` provides ``bounds`` (float64) and ``normalized_power``
    (complex128, (intervals, degree + 1, 2)), as the reference's ``KernelTable`` does."""
    if table is None:
        return None
    obs_pts, src_pts = _double(obs_pts), _double(src_pts)
    weights, phi = _double(weights), _double(phi)
    obs_normals, src_normals = _double(obs_normals), _double(src_normals)
    far = np.ascontiguousarray(far, dtype=np.uint8)
    mb, q = obs_pts.shape[:2]
    nb, width = src_pts.shape[0], phi.shape[1]
    if (obs_pts.shape != (mb, q, 2) or src_pts.shape != (nb, q, 2) or weights.shape != (q,) or
            phi.shape != (q, width) or obs_normals.shape != (mb, 2) or src_normals.shape != (nb, 2) or
            far.shape != (mb, nb)):
        raise ValueError('Invalid far-block layout.')
    bounds = np.ascontiguousarray(table.bounds, dtype=np.float64)
    coeff = np.ascontiguousarray(table.normalized_power, dtype=np.complex128)
    if coeff.ndim != 3 or coeff.shape[0] != len(bounds) - 1 or coeff.shape[2] != 2:
        raise ValueError('Invalid kernel-table layout.')
    k = complex(k)

    def buffer(wanted):
        return np.zeros((width * width, mb, nb), dtype=np.complex128) if wanted else None
    acc_s, acc_k, acc_kt = buffer(want_s), buffer(want_k), buffer(want_k and mirrored)
    lib = _lib.load()
    status = lib.ghost_far_block(mb, nb, q, width, obs_pts.ctypes.data, src_pts.ctypes.data, weights.ctypes.data,
                                 phi.ctypes.data, obs_normals.ctypes.data, src_normals.ctypes.data, far.ctypes.data,
                                 int(bool(obs_normal_deriv)), int(bool(want_s)), int(bool(want_k)),
                                 int(bool(mirrored)), k.real, k.imag, len(bounds) - 1, bounds.ctypes.data,
                                 coeff.shape[1] - 1, coeff.ctypes.data,
                                 *(None if a is None else a.ctypes.data for a in (acc_s, acc_k, acc_kt)))
    if status == 2:
        return None
    if status == 3:
        raise RuntimeError('Far-block quadrature rejected its inputs.')
    _lib.check(status, 'ghost_far_block')
    return acc_s, acc_k, acc_kt


class KernelTable:
    """Piecewise-polynomial table of G = (j/4) H0^(2)(kr) and dG = (j/4) k H1^(2)(kr) in the
    layout ``far_block`` reads (``bounds``; ``normalized_power`` (intervals, degree + 1, 2):
    ascending powers of the interval coordinate x in [0, 1], channels G and dG).  Built by
    Chebyshev interpolation at degree + 1 points per interval, intervals about 1/4
    wavelength long above r = 1/|k| and geometric below, the same kind of table as the
    reference's ``twod/assembly/kernels.py:337`` (whose builder and checks are its own)."""

    def __init__(self, k, upper, degree=12, lower=5e-13):
        from numpy.polynomial import chebyshev as C
        from scipy.special import hankel2
        k = complex(k)
        ka = abs(k)
        b = [lower]
        while b[-1] < upper:
            r = b[-1]
            step = min(r, 0.25 / ka) if r < 1.0 / ka else 0.25 * 2 * np.pi / ka / 4
            b.append(min(upper, r + max(step, 1e-14)))
        self.bounds = np.array(b)
        n = degree + 1
        x = np.cos(np.pi * (np.arange(n) + 0.5) / n)
        lo, width = self.bounds[:-1, None], np.diff(self.bounds)[:, None]
        rr = lo + (x + 1) * 0.5 * width
        vals = np.stack([0.25j * hankel2(0, k * rr), 0.25j * k * hankel2(1, k * rr)], axis=-1)
        power = np.zeros((len(lo), n, 2), complex)
        # Chebyshev fit in t in [-1, 1], then convert to powers of x = (t + 1) / 2
        for c in range(2):
            for i in range(len(lo)):
                cheb = C.chebfit(x, vals[i, :, c], degree)
                poly_t = C.cheb2poly(cheb)
                px = _compose(poly_t)  # p(t) with t = 2x - 1
                power[i, :len(px), c] = px
        self.normalized_power = np.ascontiguousarray(power)


def _compose(poly_t):
    """Coefficients in x of p(2x - 1) for p given by ascending coefficients in t."""
    out = np.zeros(len(poly_t), complex)
    term = np.array([1.0 + 0j])
    lin = np.array([-1.0, 2.0])
    for c in poly_t:
        out[:len(term)] += c * term
        term = np.convolve(term, lin)
    return out
