"""Linear-Galerkin combined-field solve of closed PEC contours on the device.

This is the reference's own 2-D discretisation of a closed perfectly conducting contour
in air (``twod/formulations/combined_regions.py:21-62``, ``twod/solver.py:1828-1840``):
straight elements with linear (hat) bases, one unknown per node, and the combined rows

* TM (Dirichlet trace): ``S + gamma (D + M/2)``, right-hand side ``-load``;
* TE (flux): ``K' - M/2 - gamma W``, right-hand side ``-(normal-derivative load)``;

with ``gamma = 1/(j k)``, which keep both channels free of the interior resonances of the
closed body.  Every arithmetic step runs in libgrimgpu (``grim_gal_*``): the near-pair
structure (built once per mesh), the near and far element-pair blocks, the routing and
the node gather, the plane-wave loads and the far field.

Node order follows the reference's solver: each drawn (clockwise) contour is reversed
about its first point (``twod/geometry.py:1009`` ``_apply_user_convention_flip``), element
j runs from node j to node j + 1, its normal is (-t_y, t_x) (``twod/geometry.py:1935``).
"""
from __future__ import annotations

import ctypes

import os

import numpy as np
import torch

from .. import _lib
from ..device import context, ptr

W_FAR_FLOOR = 8        # calibrated far order of the W blocks (linear elements)
FAR_CAP = 8            # the reference's default far order, reduced only by its calibrated table


def solver_contour(drawn):
    """Nodes of a drawn closed contour in the reference solver's order (reversed about its
    first point)."""
    drawn = np.asarray(drawn, dtype=np.float64)
    return drawn[(-np.arange(len(drawn))) % len(drawn)]


def element_arrays(polygons):
    """(elem (ne, 8), nodes (ne, 2) int32, start_of (n,), end_of (n,)) of closed contours
    given as drawn vertex arrays.  elem rows: start point, end point, unit normal
    (-t_y, t_x), length, 0."""
    elems, nodes, start_of, end_of = [], [], [], []
    base = 0
    for drawn in polygons:
        pts = solver_contour(drawn)
        m = len(pts)
        if m < 3:
            raise ValueError('A closed contour needs at least three vertices.')
        a, b = pts, np.roll(pts, -1, axis=0)
        d = b - a
        length = np.hypot(d[:, 0], d[:, 1])
        if np.any(length <= 0.0):
            raise ValueError('Zero-length element.')
        t = d / length[:, None]
        elems.append(np.column_stack([a, b, -t[:, 1], t[:, 0], length, np.zeros(m)]))
        idx = base + np.arange(m)
        nodes.append(np.stack([idx, base + (np.arange(m) + 1) % m], axis=1))
        start_of.append(idx)
        end_of.append(base + (np.arange(m) - 1) % m)
        base += m
    cat = np.concatenate
    return (np.ascontiguousarray(cat(elems)), np.ascontiguousarray(cat(nodes), dtype=np.int32),
            np.ascontiguousarray(cat(start_of), dtype=np.int32), np.ascontiguousarray(cat(end_of), dtype=np.int32))


def w_far_order(k, lengths):
    """The reference's far Gauss order of the TE rows (``twod/operators.py:1512``
    ``_graded_w_far_floor`` and ``:2433``): 8 when 1e-4 <= |k| L_max <= 3 and no element is
    shorter than 0.001 L_max (the W rule's calibration), else 16; never below the caller's 8."""
    longest = float(np.max(lengths))
    calibrated = 1e-4 <= abs(float(k)) * longest <= 3.0 and float(np.min(lengths)) >= 1e-3 * longest
    return max(W_FAR_FLOOR if calibrated else 16, FAR_CAP)


class GalerkinBody:
    """Element geometry and near-pair structure of closed contours, resident in HBM.

    The near-pair list depends on the geometry only, so it is built once here (one
    stream synchronisation to size it) and reused by every fill of every wavenumber and
    polarisation."""

    def __init__(self, polygons, device=None, ctx=None):
        ctx = ctx or context()
        elem, nodes, start_of, end_of = element_arrays(polygons)
        dev = device or torch.device('cuda', torch.cuda.current_device())
        self.ne = int(elem.shape[0])
        self.n = int(start_of.shape[0])
        self.lengths = elem[:, 6].copy()
        self.elem = torch.from_numpy(elem).to(dev)
        self.nodes = torch.from_numpy(nodes).to(dev)
        self.start_of = torch.from_numpy(start_of).to(dev)
        self.end_of = torch.from_numpy(end_of).to(dev)
        self.geom = self.elem  # device of the body (the pipeline reads body.geom.device)
        self.h2d_bytes = elem.nbytes + nodes.nbytes + start_of.nbytes + end_of.nbytes
        self.row_off = torch.empty(self.ne + 1, dtype=torch.int32, device=dev)
        nnz = ctypes.c_int(0)
        _lib.check(ctx.lib.grim_gal_near_count(ctx.h, self.ne, ptr(self.elem), ptr(self.nodes), ptr(self.row_off),
                                               ctypes.byref(nnz)), 'grim_gal_near_count')
        self.nnz = int(nnz.value)
        self.col = torch.empty(max(1, self.nnz), dtype=torch.int32, device=dev)
        self.route = torch.empty(max(1, self.nnz), dtype=torch.int32, device=dev)
        _lib.check(ctx.lib.grim_gal_near_list(ctx.h, self.ne, ptr(self.elem), ptr(self.nodes), ptr(self.row_off),
                                              ptr(self.col), ptr(self.route)), 'grim_gal_near_list')
        # the adaptive (route 3) pairs get a CTA each: their indices, in list order
        routes = self.route[:self.nnz].cpu().numpy()
        adapt = np.flatnonzero(routes == 3).astype(np.int32)
        self.nadapt = int(adapt.size)
        self.adapt_idx = torch.from_numpy(adapt if adapt.size else np.zeros(1, np.int32)).to(dev)
        self.route_counts = np.bincount(routes, minlength=4)

    # partial pivoting leaves the diagonal on these systems (and unpivoted elimination grows
    # by up to 1e10 on cosine-spaced airfoils): their factorizations pivot throughout, with
    # LAPACK's partial pivoting (GRIM_GALERKIN_PIVOT=tournament selects tournament pivoting)
    pivot = 'tournament' if os.environ.get('GRIM_GALERKIN_PIVOT', 'partial') == 'tournament' else 'partial'

    def far_min_order(self, k, pol):
        return w_far_order(k, self.lengths) if pol == 'TE' else 0

    def fill_matrix(self, k, pol, complex64=False, out=None, ctx=None):
        """Combined-field node matrix (column-major in an (n, n) tensor)."""
        ctx = ctx or context()
        n = self.n
        dt = torch.complex64 if complex64 else torch.complex128
        z = out if out is not None else torch.empty((n, n), dtype=dt, device=self.elem.device)
        _lib.check(ctx.lib.grim_gal_fill(ctx.h, _lib.POL_TM if pol == 'TM' else _lib.POL_TE, self.ne, n,
                                         ptr(self.elem), ptr(self.nodes), ptr(self.start_of), ptr(self.end_of),
                                         ptr(self.row_off), ptr(self.col), ptr(self.route), self.nnz,
                                         ptr(self.adapt_idx), self.nadapt, float(k),
                                         int(self.far_min_order(k, pol)), ptr(z), n, int(complex64)), 'grim_gal_fill')
        return z

    def rhs_matrix(self, k, pol, angles_dev, complex64=False, out=None, ctx=None):
        ctx = ctx or context()
        n, nang = self.n, int(angles_dev.numel())
        dt = torch.complex64 if complex64 else torch.complex128
        b = out if out is not None else torch.empty((nang, n), dtype=dt, device=self.elem.device)
        _lib.check(ctx.lib.grim_gal_rhs(ctx.h, _lib.POL_TM if pol == 'TM' else _lib.POL_TE, n, ptr(self.elem),
                                        ptr(self.start_of), ptr(self.end_of), nang, ptr(angles_dev), float(k), ptr(b),
                                        n, int(complex64)), 'grim_gal_rhs')
        return b

    def far_amplitude(self, k, angles_dev, x, out=None, ctx=None):
        ctx = ctx or context()
        nang = int(angles_dev.numel())
        amp = out if out is not None else torch.empty(nang, dtype=torch.complex128, device=self.elem.device)
        _lib.check(ctx.lib.grim_gal_farfield(ctx.h, self.ne, ptr(self.elem), ptr(self.nodes), nang, ptr(angles_dev),
                                             float(k), ptr(x), self.n, int(x.dtype == torch.complex64), ptr(amp)),
                   'grim_gal_farfield')
        return amp

    def check_status(self, ctx=None):
        """Raise FloatingPointError when a near-pair rule of a fill on this handle failed
        (the reference raises the same for an unconverged close pair)."""
        ctx = ctx or context()
        flag = ctypes.c_int(0)
        _lib.check(ctx.lib.grim_gal_status(ctx.h, ctypes.byref(flag)), 'grim_gal_status')
        if flag.value:
            raise FloatingPointError('close-pair quadrature did not converge')


def sigma_from_amplitude(amp, k):
    """sigma_2D = |amp|^2 / (4 k) (``twod/solver.py:838``)."""
    return 0.25 / float(k) * np.abs(np.asarray(amp)) ** 2

