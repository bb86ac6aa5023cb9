"""FP64 oracle: pulse-basis, point-matched 2-D TM EFIE / TE MFIE (test infrastructure).

This is the checker for the GPU fill, excitation, solve and far-field kernels.  It
follows the reference's conventions (``ghost_backend`` = ``tools/GHOST/ghost_backend``):

* time convention exp(+j w t); outgoing Hankel H^(2); incident field
  u_inc = exp(+j k d.r) with d = (cos phi, sin phi) and the "coming-from" angle
  phi (0 deg arrives from the right) -- ``twod/assembly/kernels.py:223-294``,
  ``twod/solver.py:2027-2030``;
* single-layer kernel S(r, r') = (j/4) H0^(2)(k|r - r'|) -- ``twod/operators.py:1577``
  (``_far_green_into``) and ``twod/special.py:220``;
* stored amplitude B = sum_n sigma_n * int_n exp(+j k d.r') dl' (the SLP projection
  with the RHS plane-wave moments as weights, ``twod/assembly/kernels.py:163-191``),
  sigma_2D = |B|^2 / (4 k) (``twod/solver.py:838-859``, ``twod/constants.py:19``),
  physical amplitude A = +j B;
* TM = HH (Dirichlet), TE = VV (Neumann) -- ``twod/solver.py:407-422``.

Formulation (pulse basis on straight panels, collocation at panel midpoints):

TM  (u = 0 on the PEC):          sum_n Z_mn s_n = -u_inc(c_m),
    Z_mn = int_n S(c_m, r') dl'.
TE  (du/dn = 0 on the PEC):      sum_n Z_mn s_n = -du_inc/dn(c_m) = -j k (d.n_m) u_inc(c_m),
    Z_mm = 1/2 (exterior jump of the normal derivative of the S layer, outward n),
    Z_mn = int_n dS/dn_m dl' = -(k/4) (Y1 + j J1)(kR) (Rhat . n_m),  Rhat = (c_m - r')/R.

Off-diagonal entries use Gauss-Legendre rules on the source panel whose order
depends on the normalised distance delta = dist(c_m, panel n) / h_n (h_n the
half-length): 12 points for delta < 2, 6 for delta < 6, 4 otherwise
(``quad_order``).  The TM self term is integrated exactly by the term-wise
integrated power series of J0 and Y0 (``tm_self_term``).  The GPU kernels use the
same rules, so GPU-vs-oracle differences are rounding only.
"""
from __future__ import annotations

import math

import numpy as np
from scipy import special as sp

EULER_GAMMA = 0.5772156649015329
QUAD_NEAR_DELTA = 2.0
QUAD_MID_DELTA = 6.0
QUAD_ORDERS = (12, 6, 4)


def gauss_legendre(q):
    x, w = np.polynomial.legendre.leggauss(int(q))
    return x, w


def panel_arrays(vertices_list):
    """Closed polygons -> panel arrays (centers, tangents, half-lengths, outward normals).

    ``vertices_list``: list of (N_i, 2) arrays, each a closed polygon listed without
    repeating the first vertex.  Orientation is detected from the signed area, so
    clockwise (the reference's required order) and counter-clockwise both work.
    """
    centers, tangents, halves, normals = [], [], [], []
    for v in vertices_list:
        v = np.asarray(v, dtype=np.float64)
        a = v
        b = np.roll(v, -1, axis=0)
        area = 0.5 * np.sum(a[:, 0] * b[:, 1] - b[:, 0] * a[:, 1])
        edge = b - a
        length = np.hypot(edge[:, 0], edge[:, 1])
        t = edge / length[:, None]
        s = 1.0 if area < 0.0 else -1.0
        n = s * np.stack([-t[:, 1], t[:, 0]], axis=1)
        centers.append(0.5 * (a + b))
        tangents.append(t)
        halves.append(0.5 * length)
        normals.append(n)
    return (np.concatenate(centers), np.concatenate(tangents),
            np.concatenate(halves), np.concatenate(normals))


CORNER_TURN_RAD = math.radians(20.0)


def te_curvature_correction(vertices_list):
    """Per-panel TE self-term correction kappa_bar * L / (4 pi).

    A straight self panel drops the smooth-curve diagonal limit kappa/(4 pi) of the
    normal-derivative kernel over the panel's own arc.  The curvature of the curve
    the polygon samples is estimated at each vertex as the turning angle over the
    mean adjacent panel length, kappa_v = beta_v / ((L_prev + L_next)/2) (convex
    turns positive); vertices that turn by more than 20 degrees are treated as
    true corners (kappa_v = 0).  Panel i gets (kappa_i + kappa_{i+1})/2 * L_i/(4 pi).
    """
    out = []
    for v in vertices_list:
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
        kappa = np.where(np.abs(beta) <= CORNER_TURN_RAD, beta / (0.5 * (lp + length)), 0.0)
        out.append(0.5 * (kappa + np.roll(kappa, -1)) * length / (4.0 * math.pi))
    return np.concatenate(out)


def point_segment_distance(p, c, t, h):
    """Distance from points p (M,2) to segments (c, t, h) (N,...) -> (M, N)."""
    dx = p[:, None, 0] - c[None, :, 0]
    dy = p[:, None, 1] - c[None, :, 1]
    along = dx * t[None, :, 0] + dy * t[None, :, 1]
    clamped = np.clip(along, -h[None, :], h[None, :])
    ex = dx - clamped * t[None, :, 0]
    ey = dy - clamped * t[None, :, 1]
    return np.hypot(ex, ey)


def quad_order(delta):
    q = np.full(delta.shape, QUAD_ORDERS[2], dtype=np.int64)
    q[delta < QUAD_MID_DELTA] = QUAD_ORDERS[1]
    q[delta < QUAD_NEAR_DELTA] = QUAD_ORDERS[0]
    return q


def integral_j0_y0(x):
    """(int_0^x J0(u) du, int_0^x Y0(u) du) by the term-wise integrated series.

    J0(u) = sum_s c_s (u)^{2s},  c_s = (-1)^s / (4^s (s!)^2)
    Y0(u) = (2/pi) [ln(u/2) + gamma] J0(u) - (2/pi) sum_{s>=1} c_s H_s u^{2s}
    (DLMF 10.8.2), and int_0^x u^{2s} ln(u/2) du = x^{2s+1}/(2s+1) [ln(x/2) - 1/(2s+1)].
    """
    x = float(x)
    lx = math.log(0.5 * x)
    ij = 0.0
    iy = 0.0
    c = 1.0
    harm = 0.0
    p = x  # x^{2s+1}
    for s in range(0, 200):
        if s > 0:
            c *= -1.0 / (4.0 * s * s)
            harm += 1.0 / s
            p *= x * x
        term = c * p / (2 * s + 1)
        ij += term
        iy += term * (lx + EULER_GAMMA - 1.0 / (2 * s + 1) - harm)
        if s > 4 and abs(term) * (1.0 + abs(lx) + harm) < 1e-18 * max(1.0, abs(ij)):
            break
    return ij, (2.0 / math.pi) * iy


def tm_self_term(k, h):
    """int_{-h}^{h} (j/4) H0^(2)(k|t|) dt = (j/(2k)) int_0^{kh} (J0 - j Y0) du."""
    ij, iy = integral_j0_y0(k * h)
    return (1j / (2.0 * k)) * complex(ij, -iy)


def _kernel_tm(k, r):
    kr = k * r
    return 0.25 * (sp.y0(kr) + 1j * sp.j0(kr))


def _kernel_te(k, r, rdotn):
    kr = k * r
    return -0.25 * k * (sp.y1(kr) + 1j * sp.j1(kr)) * rdotn


def fill(k, centers, tangents, halves, normals, polarization, rows=None, te_diag=None):
    """Dense system matrix Z (complex128, shape (M, N)); ``rows`` selects observation panels.

    ``te_diag`` (TE only): per-panel real addition to the 1/2 diagonal
    (``te_curvature_correction``).
    """
    pol = polarization.upper()
    n_all = len(centers)
    rows = np.arange(n_all) if rows is None else np.asarray(rows)
    obs = centers[rows]
    nrm = normals[rows]
    delta = point_segment_distance(obs, centers, tangents, halves) / halves[None, :]
    q = quad_order(delta)
    z = np.zeros((len(rows), n_all), dtype=np.complex128)
    for qq in sorted(set(q.ravel().tolist())):
        xg, wg = gauss_legendre(qq)
        mask = q == qq
        mi, ni = np.nonzero(mask)
        acc = np.zeros(len(mi), dtype=np.complex128)
        for xq, wq in zip(xg, wg):
            sx = centers[ni, 0] + xq * halves[ni] * tangents[ni, 0]
            sy = centers[ni, 1] + xq * halves[ni] * tangents[ni, 1]
            dx = obs[mi, 0] - sx
            dy = obs[mi, 1] - sy
            r = np.hypot(dx, dy)
            if pol == 'TM':
                val = _kernel_tm(k, r)
            else:
                rdotn = (dx * nrm[mi, 0] + dy * nrm[mi, 1]) / r
                val = _kernel_te(k, r, rdotn)
            acc += (wq * halves[ni]) * val
        z[mi, ni] = acc
    for local, m in enumerate(rows):
        if pol == 'TM':
            z[local, m] = tm_self_term(k, halves[m])
        else:
            z[local, m] = 0.5 + (0.0 if te_diag is None else te_diag[m])
    return z


def directions(angles_deg):
    phi = np.deg2rad(np.asarray(angles_deg, dtype=np.float64))
    return np.stack([np.cos(phi), np.sin(phi)], axis=1)


def rhs(k, centers, normals, angles_deg, polarization):
    d = directions(angles_deg)
    phase = np.exp(1j * k * (centers @ d.T))
    if polarization.upper() == 'TM':
        return -phase
    return -(1j * k * (normals @ d.T)) * phase


def farfield_weights(k, centers, tangents, halves, angles_deg):
    """w_n(phi) = int_n exp(+j k d.r') dl' = 2h exp(j k d.c) sinc(k (d.t) h)."""
    d = directions(angles_deg)
    arg = k * (tangents @ d.T) * halves[:, None]
    sinc = np.where(np.abs(arg) < 1e-8, 1.0 - arg * arg / 6.0, np.sin(arg) / np.where(arg == 0, 1.0, arg))
    return (2.0 * halves[:, None]) * np.exp(1j * k * (centers @ d.T)) * sinc


def monostatic_amplitude(weights, density):
    return np.einsum('na,na->a', weights, density)


def sigma_2d(amplitude, k):
    return 0.25 / k * np.abs(amplitude) ** 2


def sigma_db(sigma, floor=1e-12):
    return 10.0 * np.log10(np.maximum(sigma, floor))


def solve(k, vertices_list, angles_deg, polarization):
    """Full FP64 monostatic solve -> dict(amplitude, sigma, density, matrix, rhs)."""
    import scipy.linalg as sla
    c, t, h, n = panel_arrays(vertices_list)
    te_diag = te_curvature_correction(vertices_list) if polarization.upper() == 'TE' else None
    z = fill(k, c, t, h, n, polarization, te_diag=te_diag)
    b = rhs(k, c, n, angles_deg, polarization)
    lu = sla.lu_factor(z, check_finite=False)
    x = sla.lu_solve(lu, b, check_finite=False)
    w = farfield_weights(k, c, t, h, angles_deg)
    amp = monostatic_amplitude(w, x)
    return dict(amplitude=amp, sigma=sigma_2d(amp, k), density=x, matrix=z, rhs=b, lu=lu)


def backward_error(a, x, b):
    """Normwise backward error per column, as ``twod/solver.py:695-720`` computes it."""
    r = a @ x - b
    ainf = np.max(np.sum(np.abs(a), axis=1))
    num = np.max(np.abs(r), axis=0)
    den = ainf * np.max(np.abs(x), axis=0) + np.max(np.abs(b), axis=0)
    return num / np.where(den > 0, den, 1.0)
