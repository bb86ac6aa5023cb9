"""CPU restatement of the reference's 2-D linear-Galerkin near element blocks (TEST INFRASTRUCTURE).

Only the tests import this module: it is the checker for a GPU port of these blocks, never a
product path.  It restates, for straight elements with linear (hat) bases and a real
wavenumber:

* the single-layer self block (``twod/operators.py:1044`` ``_single_layer_block_linear``):
  on a straight element the kernel depends on u = |t - s| only, so the 2 x 2 block is
  l^2 (j/4) int_0^1 H0^(2)(k l u) C(u) du with C_diag = (2 - 3u + u^3)/3 and
  C_off = (1 - u^3)/3; the small-argument series of H0^(2) (J0 times the log term, plus the
  harmonic-number corrections) turns it into exact moments int u^p = 1/(p+1) and
  int u^p ln u = -1/(p+1)^2 (``:418`` ``_single_layer_self_block_exact``, up to |k l| = 8);
  beyond, the element is cut into m sub-intervals with |k| l / m <= 2, each sub-interval's
  own block by the series, neighbouring sub-intervals by the graded corner rule and
  separated ones by a 16-point tensor rule, all in the parent element's basis (``:980``
  ``_single_layer_self_block_composite``);
* the S and K' blocks of endpoint-touching pairs (``:629``
  ``_integrate_linear_touching_duffy_sk_vectorized``): the unit square split into two
  triangles at the shared corner, the radial distance graded as u = t^4 (weight 4 t^7) with
  a 20-point Gauss rule per direction (``polynomial_quadrature.py:319`` ``_nodes``), the
  separations formed from the corner so that points next to it keep their accuracy;
* the routing of separated pairs (``twod/assembly/separation.py:67`` ``requires_adaptive``):
  the adaptive rule when the centres are closer than 0.75 L, the segments closer than
  0.25 L, or an end lies within 0.5 L above the other element's interior (L the longer
  length), else the fixed tensor rule;
* the fixed-rule S and K' blocks (``twod/operators.py:223``
  ``_integrate_linear_pairs_box_sk_batched``): 16 Gauss points on each element (the order
  the reference's ladder settles on for linear elements, ``operators.py:1761-1766``);
* the close separated pairs (``twod/operators.py:1172`` ``_integrate_linear_pair_adaptive_sk``):
  each box of sub-intervals compared with its four-way bisection by the same tensor rule,
  only the unconverged children refined further, to 1e-9 relative to the sum of the
  children's norms (at most 12 levels);
* the Maue hypersingular blocks from the S blocks (``:1295,1943``);
* the whole node-based S and observation-normal K' of a contour of at most 192 elements
  (``:2087`` ``_assemble_multi``, one assembly tile): far pairs (centre distance at least 3 x
  the longer length, no shared node) by the tensor rule at the tile's calibrated order
  (``:1443,1474``), near pairs by the routes above, each block added at its nodes; with the
  hypersingular W beside them (``:2799``, far S blocks at the W order ``:1512,2433``);
* the combined PEC system of a closed contour in air as the reference's dense solver receives
  it (``twod/formulations/regions.py:283-292``, ``twod/formulations/combined_regions.py:21-62,
  149-204``): S + gamma (D + M/2) for TM, K' - M/2 - gamma W for TE, gamma = 1/(j k), with
  the consistent mass M and the plane-wave loads, on the solver's reversed node order; and
  the monostatic scattering width of its solution (single- plus gamma-weighted double-layer
  far field, sigma = |amp|^2 / (4 k)).

G = (j/4) H0^(2)(k r); the normal derivative is (j/4) k H1^(2)(k r) (r . n)/r on the source
normal (negated for the observation normal); r is floored at 1e-12 and k r at 1e-12.
J0, Y0, J1, Y1 are SciPy's (the reference's own call sites, ``operators.py:898``).

Pinned against the reference's own blocks in ``tests/golden/galerkin_near.npz`` (made by
``tests/golden/make_galerkin_near_golden.py``) and its whole dense systems in
``tests/golden/ref_dense_system.npz`` (made by ``tests/golden/make_golden.py``).
"""
from __future__ import annotations

import cmath
import math

import numpy as np
from scipy import special as sp

EPS = 1e-12
EULER_GAMMA = 0.5772156649015329
SERIES_LIMIT = 8.0      # |k l| up to which the self series is used
SUBINTERVAL_KL = 2.0    # |k| l per sub-interval of the composite self rule
TOUCH_ORDER = 20        # Gauss points per direction of the graded corner rule


def unit_gauss(q):
    x, w = np.polynomial.legendre.leggauss(int(q))
    return 0.5 * (x + 1.0), 0.5 * w


def hankel2(order, x):
    """H_order^(2) at real non-negative x (floored at 1e-12)."""
    xr = np.maximum(np.asarray(x, dtype=float), 1e-12)
    if order == 0:
        return sp.j0(xr) - 1j * sp.y0(xr)
    return sp.j1(xr) - 1j * sp.y1(xr)


def green(k, r):
    """(j/4) H0^(2)(k r), r floored at EPS."""
    x = float(k) * np.maximum(np.asarray(r, dtype=float), EPS)
    return 0.25j * hankel2(0, np.where(np.abs(x) <= 1e-12, 1e-12, x))


def _moments(p, coeffs):
    """(int_0^1 u^p c(u) du, int_0^1 u^p ln(u) c(u) du) for c(u) = sum_q coeffs[q] u^q."""
    plain = sum(c / (p + q + 1) for q, c in enumerate(coeffs))
    logged = -sum(c / (p + q + 1) ** 2 for q, c in enumerate(coeffs))
    return plain, logged


def self_block_series(length, k, a=0.0, b=1.0):
    """2 x 2 single-layer block of the sub-interval [a, b] of a straight element (parent
    basis), by the small-argument series; None where |k l| is outside (1e-30, 8]."""
    ell = float(length) * (float(b) - float(a))
    if ell <= 0.0:
        return np.zeros((2, 2), dtype=np.complex128)
    z = complex(k) * ell
    if abs(z) > SERIES_LIMIT or abs(z) <= 1e-30:
        return None
    weights = {'diag': (2.0 / 3.0, -1.0, 0.0, 1.0 / 3.0), 'off': (1.0 / 3.0, 0.0, 0.0, -1.0 / 3.0)}
    c = 2.0 / math.pi
    shift = cmath.log(z / 2.0) + EULER_GAMMA
    quarter = (z / 2.0) ** 2
    total = {'diag': 0j, 'off': 0j}
    term, harmonic, m = 1.0 + 0j, 0.0, 0
    while True:
        factor = term * (1.0 - 1j * c * (shift - harmonic))
        for key, coeffs in weights.items():
            plain, logged = _moments(2 * m, coeffs)
            total[key] += factor * plain - 1j * c * term * logged
        m += 1
        term *= -quarter / (m * m)
        harmonic += 1.0 / m
        if m > 60:
            return None
        if abs(term) < 1e-18 * max(1.0, abs(total['diag'])):
            break
    block = (0.25j * ell * ell) * np.array([[total['diag'], total['off']], [total['off'], total['diag']]])
    if a == 0.0 and b == 1.0:
        return block
    t = np.array([[1.0 - a, 1.0 - b], [a, b]], dtype=np.complex128)
    return t @ block @ t.T


def touching_nodes(order=TOUCH_ORDER):
    """(x, y, w): distances from the shared corner on the unit square by two triangles, the
    radial coordinate graded as t^4."""
    n = max(int(order), TOUCH_ORDER)
    t, w = unit_gauss(n)
    u = t[:, None] ** 4
    v = t[None, :]
    wt = (4.0 * t[:, None] ** 7 * w[:, None] * w[None, :]).ravel()
    x = np.concatenate((np.broadcast_to(u, (n, n)).ravel(), (u * v).ravel()))
    y = np.concatenate(((u * v).ravel(), np.broadcast_to(u, (n, n)).ravel()))
    return x, y, np.tile(wt, 2)


def self_block_composite(length, k):
    """Self block of an electrically long straight element (|k l| > 8)."""
    ell = float(length)
    kl = abs(complex(k)) * ell
    m = max(2, int(math.ceil(kl / SUBINTERVAL_KL)))
    if m > 256:
        m = max(256, int(math.ceil(kl / SERIES_LIMIT)))
    h = 1.0 / m
    block = np.zeros((2, 2), dtype=np.complex128)
    for i in range(m):
        block += self_block_series(length, k, i * h, (i + 1) * h)

    def basis(x):
        return np.stack((1.0 - x, x), axis=-1)

    # neighbouring sub-intervals, meeting at s = (i + 1) h
    x, y, w = touching_nodes(TOUCH_ORDER)
    g = green(k, ell * h * (x + y)) * w
    joints = (np.arange(m - 1) + 1.0) * h
    for side in (-1.0, 1.0):
        xo = joints[:, None] + side * h * x[None, :]
        xs = joints[:, None] - side * h * y[None, :]
        block += np.einsum('q,iqa,iqb->ab', g, basis(xo), basis(xs)) * (ell * h) ** 2
    # separated sub-intervals: the kernel depends on the offset d only
    t, wt = unit_gauss(16)
    for d in range(2, m):
        kern = green(k, ell * h * (d + t[None, :] - t[:, None])) * np.outer(wt, wt)
        first = np.arange(m - d)[:, None]
        lower = basis((first + t[None, :]) * h)
        upper = basis((first + d + t[None, :]) * h)
        block += (np.einsum('pq,ipa,iqb->ab', kern, lower, upper)
                  + np.einsum('pq,iqa,ipb->ab', kern, upper, lower)) * (ell * h) ** 2
    return block


def self_block(length, k):
    """Single-layer self block of a straight element (the series, else the composite)."""
    out = self_block_series(length, k)
    if out is not None:
        return out
    if abs(complex(k)) * float(length) > SERIES_LIMIT:
        return self_block_composite(length, k)
    raise ValueError('self series failed below |k l| = 8')


def touching_blocks(obs_ends, src_ends, obs_normal, src_normal, obs_start, src_start, k, obs_normal_deriv,
                    order=TOUCH_ORDER):
    """(S, K') 2 x 2 blocks of two elements sharing an end (obs_start: the observation
    element's shared end is its start p0; likewise src_start)."""
    po0, po1 = (np.asarray(p, float) for p in obs_ends)
    ps0, ps1 = (np.asarray(p, float) for p in src_ends)
    lo, ls = float(np.hypot(*(po1 - po0))), float(np.hypot(*(ps1 - ps0)))
    x0, y0, w = touching_nodes(order)
    corner_o = po0 if obs_start else po1
    corner_s = ps0 if src_start else ps1
    d_o = (po1 - po0) if obs_start else (po0 - po1)
    d_s = (ps1 - ps0) if src_start else (ps0 - ps1)
    origin = corner_o - corner_s
    tiny = 64.0 * np.finfo(float).eps * max(float(np.hypot(*corner_o)), float(np.hypot(*corner_s)), lo, ls)
    if float(np.hypot(*origin)) <= tiny:
        origin = np.zeros(2)
    diff = origin[None, :] + x0[:, None] * d_o[None, :] - y0[:, None] * d_s[None, :]
    xo = x0 if obs_start else 1.0 - x0
    xs = y0 if src_start else 1.0 - y0
    bo = np.column_stack((1.0 - xo, xo))
    bs = np.column_stack((1.0 - xs, xs))
    r = np.hypot(diff[:, 0], diff[:, 1])
    s_blk = np.einsum('q,q,qa,qb->ab', w, green(k, r), bo, bs)
    live = r > EPS
    deriv = np.zeros(len(r), dtype=np.complex128)
    kr = float(k) * r[live]
    h1 = hankel2(1, np.where(np.abs(kr) <= 1e-12, 1e-12, kr))
    n = np.asarray(obs_normal if obs_normal_deriv else src_normal, float)
    proj = (diff[live] @ n) / r[live]
    deriv[live] = (0.25j * float(k)) * h1 * proj * (-1.0 if obs_normal_deriv else 1.0)
    k_blk = np.einsum('q,q,qa,qb->ab', w, deriv, bo, bs)
    return s_blk * (lo * ls), k_blk * (lo * ls)


# ---- separated near pairs (``twod/assembly/separation.py``, ``twod/operators.py:223``)
ADAPTIVE_CENTRE = 0.75      # centre distance below this many lengths: adaptive rule
ADAPTIVE_GAP = 0.25         # segments closer than this many lengths: adaptive rule
ADAPTIVE_PROJECTION = 0.5   # an end hovering over the other element this close: adaptive rule
BOX_ORDER = 16              # Gauss points per element of the fixed tensor rule


def _point_to_segment_sq(x, a, b):
    edge = b - a
    den = float(edge @ edge)
    t = float((x - a) @ edge) / den if den > 0 else 0.0
    d = x - a - min(max(t, 0.0), 1.0) * edge
    return float(d @ d)


def segment_distance(p0, p1, q0, q1):
    """Distance between two closed segments (0 when they cross)."""
    p0, p1, q0, q1 = (np.asarray(v, float) for v in (p0, p1, q0, q1))
    sq = min(_point_to_segment_sq(p0, q0, q1), _point_to_segment_sq(p1, q0, q1),
             _point_to_segment_sq(q0, p0, p1), _point_to_segment_sq(q1, p0, p1))
    u, v, w = p1 - p0, q1 - q0, q0 - p0
    cross = lambda a, b: a[0] * b[1] - a[1] * b[0]
    den = cross(u, v)
    if den != 0:
        t, s = cross(w, v) / den, cross(w, u) / den
        if 0 <= t <= 1 and 0 <= s <= 1:
            return 0.0
    return math.sqrt(max(sq, 0.0))


def projection_distance(p0, p1, q0, q1):
    """Smallest distance from an end of one segment to the other's interior (its foot point
    strictly inside), infinity when no end projects inside."""
    p0, p1, q0, q1 = (np.asarray(v, float) for v in (p0, p1, q0, q1))
    best = math.inf
    for x, a, b in ((p0, q0, q1), (p1, q0, q1), (q0, p0, p1), (q1, p0, p1)):
        edge = b - a
        den = float(edge @ edge)
        t = float((x - a) @ edge) / den if den > 0 else -1.0
        if 0.0 < t < 1.0:
            d = x - a - t * edge
            best = min(best, math.sqrt(float(d @ d)))
    return best


def needs_adaptive(obs_ends, src_ends):
    """True when a separated pair takes the adaptive rule rather than the 16-point tensor rule:
    centres closer than 0.75 L, segments closer than 0.25 L, or an end within 0.5 L above the
    other element's interior (L the longer length)."""
    p0, p1 = (np.asarray(v, float) for v in obs_ends)
    q0, q1 = (np.asarray(v, float) for v in src_ends)
    lo, ls = float(np.hypot(*(p1 - p0))), float(np.hypot(*(q1 - q0)))
    scale = max(lo, ls)
    dist = float(np.hypot(*(0.5 * (p0 + p1) - 0.5 * (q0 + q1))))
    if dist < ADAPTIVE_CENTRE * scale:
        return True
    if dist >= 0.5 * (lo + ls) + ADAPTIVE_PROJECTION * scale:
        return False
    if dist < 0.5 * (lo + ls) + ADAPTIVE_GAP * scale and segment_distance(p0, p1, q0, q1) < ADAPTIVE_GAP * scale:
        return True
    return projection_distance(p0, p1, q0, q1) < ADAPTIVE_PROJECTION * scale


def box_blocks(obs_ends, src_ends, obs_normal, src_normal, k, obs_normal_deriv, order=BOX_ORDER):
    """(S, K') 2 x 2 blocks of a separated pair by the tensor Gauss rule (order points on each
    element)."""
    p0, p1 = (np.asarray(v, float) for v in obs_ends)
    q0, q1 = (np.asarray(v, float) for v in src_ends)
    t, w = unit_gauss(order)
    basis = np.column_stack((1.0 - t, t))
    op = p0[None, :] + t[:, None] * (p1 - p0)[None, :]
    sp_ = q0[None, :] + t[:, None] * (q1 - q0)[None, :]
    diff = op[:, None, :] - sp_[None, :, :]
    r = np.sqrt(np.sum(diff * diff, axis=2))
    rs = np.maximum(r, EPS)
    kr = float(k) * rs
    ww = np.outer(w, w)
    g = 0.25 * sp.y0(kr) + 0.25j * sp.j0(kr)
    s_blk = basis.T @ (ww * g) @ basis
    deriv = 0.25 * float(k) * sp.y1(kr) + 0.25j * float(k) * sp.j1(kr)
    n = np.asarray(obs_normal if obs_normal_deriv else src_normal, float)
    proj = np.sum(diff * n[None, None, :], axis=2) / rs
    dk = (-deriv if obs_normal_deriv else deriv) * proj
    dk[r <= EPS] = 0.0
    k_blk = basis.T @ (ww * dk) @ basis
    scale = float(np.hypot(*(p1 - p0))) * float(np.hypot(*(q1 - q0)))
    return s_blk * scale, k_blk * scale


# ---- close separated pairs: bisection to a relative tolerance (``twod/operators.py:1172``)
ADAPTIVE_RTOL = 1e-9
ADAPTIVE_MAX_DEPTH = 12


def interval_box(obs_ends, src_ends, obs_normal, src_normal, k, obs_normal_deriv, obs_iv, src_iv, order=BOX_ORDER):
    """(S, K') of the sub-intervals obs_iv x src_iv (parent parameters in [0, 1]) in the
    parent elements' hat basis, by the tensor Gauss rule."""
    p0, p1 = (np.asarray(v, float) for v in obs_ends)
    q0, q1 = (np.asarray(v, float) for v in src_ends)
    (oa, ob), (sa, sb) = obs_iv, src_iv
    ho, hs = max(ob - oa, 0.0), max(sb - sa, 0.0)
    lo = float(np.hypot(*(p1 - p0))) * ho
    ls = float(np.hypot(*(q1 - q0))) * hs
    if lo <= 0.0 or ls <= 0.0:
        return np.zeros((2, 2), complex), np.zeros((2, 2), complex)
    t, w = unit_gauss(order)
    xo, xs = oa + ho * t, sa + hs * t
    bo, bs = np.column_stack((1.0 - xo, xo)), np.column_stack((1.0 - xs, xs))
    ro = p0[None, :] + xo[:, None] * (p1 - p0)[None, :]
    rsrc = q0[None, :] + xs[:, None] * (q1 - q0)[None, :]
    diff = ro[:, None, :] - rsrc[None, :, :]
    r = np.sqrt(np.sum(diff * diff, axis=2))
    rs = np.maximum(r, EPS)
    kr = float(k) * rs
    kr = np.where(np.abs(kr) <= 1e-12, 1e-12, kr)
    ww = np.outer(w, w)
    g = 0.25j * hankel2(0, kr)
    n = np.asarray(obs_normal if obs_normal_deriv else src_normal, float)
    proj = np.sum(diff * n[None, None, :], axis=2) / rs
    dk = (0.25j * float(k)) * hankel2(1, kr) * proj * (-1.0 if obs_normal_deriv else 1.0)
    dk[r <= EPS] = 0.0
    s_blk = np.einsum('ij,ia,jb->ab', ww * g, bo, bs)
    k_blk = np.einsum('ij,ia,jb->ab', ww * dk, bo, bs)
    return s_blk * (lo * ls), k_blk * (lo * ls)


def adaptive_blocks(obs_ends, src_ends, obs_normal, src_normal, k, obs_normal_deriv, order=BOX_ORDER,
                    rtol=ADAPTIVE_RTOL, max_depth=ADAPTIVE_MAX_DEPTH):
    """(S, K') of a close separated pair: each box is compared with its four-way bisection,
    and only the children whose parent did not meet rtol (relative to the sum of the
    children's norms) are refined further."""
    p0, p1 = (np.asarray(v, float) for v in obs_ends)
    q0, q1 = (np.asarray(v, float) for v in src_ends)
    floor = np.finfo(float).eps * max(1.0, float(np.hypot(*(p1 - p0))) * float(np.hypot(*(q1 - q0))))

    def box(oi, si):
        return interval_box(obs_ends, src_ends, obs_normal, src_normal, k, obs_normal_deriv, oi, si, order)

    def err(coarse, kids):
        fine = sum(kids, np.zeros((2, 2), complex))
        norms = sum(float(np.linalg.norm(b)) for b in kids)
        return float(np.linalg.norm(fine - coarse)) / max(norms, floor)

    def refine(oi, si, depth, coarse):
        om, sm = 0.5 * (oi[0] + oi[1]), 0.5 * (si[0] + si[1])
        quads = [((oi[0], om), (si[0], sm)), ((oi[0], om), (sm, si[1])),
                 ((om, oi[1]), (si[0], sm)), ((om, oi[1]), (sm, si[1]))]
        kids = [box(a, b) for a, b in quads]
        e = max(err(coarse[0], [c[0] for c in kids]), err(coarse[1], [c[1] for c in kids]))
        if e <= rtol:
            return (sum((c[0] for c in kids), np.zeros((2, 2), complex)),
                    sum((c[1] for c in kids), np.zeros((2, 2), complex)))
        if depth >= max_depth:
            raise FloatingPointError('close-pair quadrature did not converge')
        s_tot, k_tot = np.zeros((2, 2), complex), np.zeros((2, 2), complex)
        for (a, b), c in zip(quads, kids):
            cs, ck = refine(a, b, depth + 1, c)
            s_tot += cs
            k_tot += ck
        return s_tot, k_tot

    whole = ((0.0, 1.0), (0.0, 1.0))
    return refine(whole[0], whole[1], 0, box(*whole))


def maue_block(s_block, k, obs_normal, src_normal, obs_length, src_length):
    """Hypersingular 2 x 2 block from the single-layer block by the Maue identity
    (``twod/operators.py:1295,1943``): W = -k^2 (n_o . n_s) S + [[1, -1], [-1, 1]] sum(S) / (L_o L_s),
    the second term the product of the hat functions' tangential derivatives."""
    s_block = np.asarray(s_block, dtype=np.complex128)
    ndn = float(np.dot(np.asarray(obs_normal, float), np.asarray(src_normal, float)))
    total = (s_block[0, 0] + s_block[0, 1]) + (s_block[1, 0] + s_block[1, 1])
    denom = max(float(obs_length) * float(src_length), EPS * EPS)
    quotient = complex(total.real / denom, total.imag / denom)
    outer = np.array([[1.0, -1.0], [-1.0, 1.0]], dtype=np.complex128)
    return (-(complex(k) ** 2) * ndn) * s_block + outer * quotient


# ---- whole node-based operators of a closed contour (``twod/operators.py:2087`` ``_assemble_multi``)
FAR_RATIO = 3.0          # far pairs: centre distance >= 3 x the longer length, no shared node
FAR_CAP = 8              # the caller's far order, reduced only where the calibrated table allows
FAR_ORDER_TABLE = (      # (|k| L_max bound, (near, mid, far) orders for linear elements)
    (0.15, (7, 6, 5)),
    (0.50, (7, 6, 5)),
    (1.50, (7, 6, 6)),
    (3.00, (8, 8, 8)),
)


def far_order(kl_max, ratio_min, cap=FAR_CAP):
    """Gauss order of a tile whose worst far pair has these parameters
    (``twod/operators.py:1474`` ``_graded_far_order``, real k, linear elements): near / mid /
    far columns for the smallest centre-distance ratio below 5, below 10, and beyond."""
    if not float(ratio_min) >= FAR_RATIO:
        return int(cap)
    for bound, (near, mid, far) in FAR_ORDER_TABLE:
        if kl_max <= bound:
            order = near if ratio_min < 5.0 else (mid if ratio_min < 10.0 else far)
            return max(2, min(int(cap), int(order)))
    return int(cap)


W_FAR_FLOOR = 8          # calibrated W far order for linear elements; 16 outside the calibration


def w_far_order(k, lengths, order):
    """Gauss order of the far tiles that feed W (``twod/operators.py:1512`` ``_graded_w_far_floor``
    and ``:2433``): the tile's own order raised to the caller's 8 points and to the calibrated W
    floor, which is 8 for 1e-4 <= |k| L_max <= 3 with no element shorter than 0.001 L_max, else 16."""
    longest = float(np.max(lengths))
    calibrated = 1e-4 <= abs(complex(k)) * longest <= 3.0 and float(np.min(lengths)) >= 1e-3 * longest
    return max(int(order), W_FAR_FLOOR if calibrated else 16, FAR_CAP)


def mass_matrix(ends, node_ids, n_nodes):
    """Consistent linear boundary mass, L [[1/3, 1/6], [1/6, 1/3]] per element at its nodes
    (``twod/operators.py:3032`` ``_linear_mass_block``, ``twod/assembly/mass.py:6``)."""
    M = np.zeros((n_nodes, n_nodes), dtype=np.complex128)
    for (a, b), nd in zip(ends, node_ids):
        length = float(np.hypot(*(np.asarray(b, float) - np.asarray(a, float))))
        blk = length * np.array([[1.0 / 3.0, 1.0 / 6.0], [1.0 / 6.0, 1.0 / 3.0]])
        for i in range(2):
            for j in range(2):
                M[nd[i], nd[j]] += blk[i, j]
    return M


def assemble_single_tile(ends, node_ids, normals, k, n_nodes, hypersingular=False):
    """Node-based single-layer S and observation-normal K' of straight elements (at most 192,
    which the reference assembles as one tile with one far order): far pairs by the graded
    tensor rule, near pairs by the self / touching / adaptive / fixed-rule routes, each 2 x 2
    block added at its elements' node rows and columns.  With ``hypersingular`` the
    hypersingular W is returned as well: the Maue block of every element pair's S block, the
    far pairs' S blocks taken at the W far order (``twod/operators.py:2799``)."""
    ends = [tuple(np.asarray(p, float) for p in e) for e in ends]
    ne = len(ends)
    lengths = np.array([float(np.hypot(*(b - a))) for a, b in ends])
    centres = np.array([0.5 * (a + b) for a, b in ends])
    S = np.zeros((n_nodes, n_nodes), dtype=np.complex128)
    K = np.zeros((n_nodes, n_nodes), dtype=np.complex128)
    W = np.zeros((n_nodes, n_nodes), dtype=np.complex128)
    dist = np.hypot(centres[:, None, 0] - centres[None, :, 0], centres[:, None, 1] - centres[None, :, 1])
    ratio = dist / np.maximum(np.maximum(lengths[:, None], lengths[None, :]), EPS)
    shares = np.array([[bool(set(node_ids[e]) & set(node_ids[f])) for f in range(ne)] for e in range(ne)])
    far = (ratio >= FAR_RATIO) & ~shares & ~np.eye(ne, dtype=bool)
    order = far_order(abs(complex(k)) * float(lengths.max()), float(np.min(ratio[far])) if far.any() else np.inf)
    w_order = w_far_order(k, lengths, order)
    for e in range(ne):
        for f in range(ne):
            if far[e, f]:
                s_blk, k_blk = box_blocks(ends[e], ends[f], normals[e], normals[f], k, True, order=max(2, order))
            elif e == f:
                s_blk, k_blk = self_block(lengths[e], k), np.zeros((2, 2), complex)
            elif shares[e, f]:
                obs_start = node_ids[e][0] in node_ids[f]
                src_start = node_ids[f][0] in node_ids[e]
                s_blk, k_blk = touching_blocks(ends[e], ends[f], normals[e], normals[f], obs_start, src_start, k,
                                               True)
            elif needs_adaptive(ends[e], ends[f]):
                s_blk, k_blk = adaptive_blocks(ends[e], ends[f], normals[e], normals[f], k, True)
            else:
                s_blk, k_blk = box_blocks(ends[e], ends[f], normals[e], normals[f], k, True)
            rows, cols = node_ids[e], node_ids[f]
            if hypersingular:
                s_w = (box_blocks(ends[e], ends[f], normals[e], normals[f], k, True, order=w_order)[0]
                       if far[e, f] else s_blk)
                w_blk = maue_block(s_w, k, normals[e], normals[f], lengths[e], lengths[f])
            for a in range(2):
                for b in range(2):
                    S[rows[a], cols[b]] += s_blk[a, b]
                    K[rows[a], cols[b]] += k_blk[a, b]
                    if hypersingular:
                        W[rows[a], cols[b]] += w_blk[a, b]
    return (S, K, W) if hypersingular else (S, K)


# ---- the combined PEC system of a closed contour (``twod/formulations/regions.py:283-292``
# base rows, ``twod/formulations/combined_regions.py:21-62,149-204`` combined routes)
def drawn_to_solver_contour(drawn_points):
    """Nodes of a closed PEC (TYPE 2) contour in the solver's order: the reference reverses
    every drawn segment (``twod/geometry.py:1009`` ``_apply_user_convention_flip``), so its
    node j is drawn point -j and its element j runs from node j to node j + 1, the stored
    normal (-t_y, t_x) (``twod/geometry.py:1935``) pointing into the conductor."""
    drawn = np.asarray(drawn_points, float)
    n = len(drawn)
    return drawn[(-np.arange(n)) % n]


def incident_loads(ends, node_ids, normals, n_nodes, k, angles_deg, order=8):
    """Galerkin loads of the plane wave exp(j k d . r), d = (cos phi, sin phi), and of its
    normal derivative j k (d . n) exp(j k d . r), at ``order`` Gauss points per element
    (``twod/operators.py`` ``_linear_element_incident_load_many`` and
    ``_linear_element_incident_dn_load_many``)."""
    t, w = unit_gauss(order)
    phi = np.radians(np.asarray(angles_deg, float))
    d = np.stack([np.cos(phi), np.sin(phi)], axis=1)
    load = np.zeros((n_nodes, len(phi)), dtype=np.complex128)
    dn_load = np.zeros_like(load)
    for (a, b), nd, nrm in zip(ends, node_ids, normals):
        a, b = np.asarray(a, float), np.asarray(b, float)
        length = float(np.hypot(*(b - a)))
        pts = a[None, :] + t[:, None] * (b - a)[None, :]
        phase = np.exp(1j * k * (pts @ d.T))                          # (points, angles)
        dn = phase * (1j * k * (d @ np.asarray(nrm, float)))[None, :]
        for i, shape in enumerate((1.0 - t, t)):
            load[nd[i]] += length * ((w * shape) @ phase)
            dn_load[nd[i]] += length * ((w * shape) @ dn)
    return load, dn_load


def pec_combined_system(nodes, k, angles_deg, polarization, operators=None):
    """The dense system the reference hands to its dense solver for a closed PEC contour in
    air (``twod/solver.py:355`` ``_solve_dense_gpu(a_eval, rhs_eval)``), its nodes in the
    solver's order.  gamma = 1/(j k) (air on the minus side, ``combined_regions.py:39``):

    * TM (Dirichlet trace rows): A = S + gamma (D + M/2), b = -load;
    * TE (flux rows): A = K' - M/2 - gamma W, b = -(normal-derivative load);

    K' with the observation normal, D the source-normal double layer, which for the
    symmetric kernel is K' transposed.  ``operators`` = (S, K', W) reuses an assembly."""
    nodes = np.asarray(nodes, float)
    n = len(nodes)
    ends = [(nodes[i], nodes[(i + 1) % n]) for i in range(n)]
    node_ids = [(i, (i + 1) % n) for i in range(n)]
    normals = []
    for a, b in ends:
        t = (b - a) / np.hypot(*(b - a))
        normals.append(np.array([-t[1], t[0]]))
    if operators is None:
        operators = assemble_single_tile(ends, node_ids, normals, k, n, hypersingular=True)
    S, Kp, W = operators
    M = mass_matrix(ends, node_ids, n)
    gamma = 1.0 / (1j * k)
    load, dn_load = incident_loads(ends, node_ids, normals, n, k, angles_deg)
    if polarization == 'TM':
        return S + gamma * (Kp.T + 0.5 * M), -load
    if polarization == 'TE':
        return Kp - 0.5 * M - gamma * W, -dn_load
    raise ValueError("polarization must be 'TM' or 'TE'")


def pec_combined_sigma(nodes, k, angles_deg, density, order=8):
    """Monostatic 2-D scattering width of the combined PEC solution ``density`` (one column
    per angle): sigma = |amp|^2 / (4 k) (``twod/solver.py:838`` ``_rcs_sigma_from_amp``,
    ``twod/constants.py:19``), amp from ``pec_combined_amplitude``."""
    return 0.25 * np.abs(pec_combined_amplitude(nodes, k, angles_deg, density, order)) ** 2 / k


def pec_combined_amplitude(nodes, k, angles_deg, density, order=8):
    """Monostatic far-field amplitude of the combined PEC solution ``density`` (one column
    per angle): amp = sum over elements of L w_q phi_i(q) rho_i exp(j k d . r_q) (single layer)
    plus the same with rho -> gamma rho and the factor j k (d . n) (double layer), d = (cos phi,
    sin phi) (``twod/operators.py`` ``_farfield_linear_density_many``, the second potential of
    ``twod/solver.py:1979`` ``exterior_double_density``)."""
    nodes = np.asarray(nodes, float)
    n = len(nodes)
    rho = np.asarray(density, dtype=np.complex128)
    t, w = unit_gauss(order)
    phi = np.radians(np.asarray(angles_deg, float))
    d = np.stack([np.cos(phi), np.sin(phi)], axis=1)
    gamma = 1.0 / (1j * k)
    amp = np.zeros(len(phi), dtype=np.complex128)
    for i in range(n):
        a, b = nodes[i], nodes[(i + 1) % n]
        length = float(np.hypot(*(b - a)))
        tangent = (b - a) / length
        normal = np.array([-tangent[1], tangent[0]])
        pts = a[None, :] + t[:, None] * (b - a)[None, :]
        phase = np.exp(1j * k * (pts @ d.T))                                  # (points, angles)
        dens = np.outer(1.0 - t, rho[i]) + np.outer(t, rho[(i + 1) % n])     # (points, angles)
        factor = 1.0 + gamma * (1j * k * (d @ normal))[None, :]
        amp += length * np.sum(w[:, None] * dens * phase * factor, axis=0)
    return amp
