"""FP64 oracle: body-of-revolution PEC EFIE / MFIE / CFIE per azimuthal mode (test infrastructure).

Only the tests import this module: it is the checker of the GPU body-of-revolution path,
never a product path.  It restates the physics and the quadrature of the reference's BoR
solver (``ghost_backend/bor``):

* generatrix (rho, z) polyline from the +z pole to the -z pole
  (``bor/kernels.py:63`` ``Generatrix``); nodal tents T_i(t) for the t- and phi-directed
  surface current, J = sum_m e^{j m phi} sum_i (a_i T_i t_hat + b_i T_i phi_hat)
  (n_dofs = 2 Nn, ``bor/solver.py:4160``);
* axis poles: the phi component is inactive and the t component is active only for
  |m| = 1, where it is tied to phi by J_phi = j m sign(t_rho) J_t
  (``bor/solver.py:2369-2440`` ``basis_mask`` / ``basis_transform``, Galerkin reduction
  Q^H Z Q);
* EFIE, time convention e^{+j w t} (``bor/solver.py:1769-1827`` ``assemble_mode``):
  Z = j k eta 2 pi [ <W.J> - (1/k^2) <div W, div J> ] with the modal Green's function
  G_n = int_{-pi}^{pi} e^{-jkR}/(4 pi R) cos(n xi) d xi,
  R^2 = (rho - rho')^2 + (z - z')^2 + 4 rho rho' sin^2(xi/2);
* MFIE (``bor/solver.py:1962`` ``assemble_mfie_mode``): Z = (1/2) M - K, with the mass
  M_ij = 2 pi int rho T_i T_j dt and K the Galerkin contraction
  2 pi sum T_i(p) rho_p w_p K^m_uv(p, q) rho_q w_q T_j(q) of the four modal brackets
  K^m_uv = int_{-pi}^{pi} F_uv(xi) e^{-j m xi} d xi (tt, ff even in xi; tf, ft odd),
  F_uv = -p(R) [W_u . (n x (J_v x R))]-type products with p(R) = (1 + jkR) e^{-jkR}/(4 pi R^3),
  test point at phi = 0, source at phi' = -xi, n = (-t_z, 0, t_rho)
  (``bor/kernels.py:896`` ``_mfie_brackets``), evaluated in the cancellation-free form
  with h = 1 - cos xi (``bor/kernels.py:996`` ``_stable_brackets``: the O(h^2) parts of
  the sampled products cancel analytically);
* CFIE (``bor/solver.py:4285-4301, 4374-4380``): Z = alpha Z_EFIE + (1 - alpha) eta0 Z_MFIE,
  V = alpha V_EFIE + (1 - alpha) eta0 V_MFIE, V_MFIE = <W, n x H_inc>
  (``bor/solver.py:2048`` ``rhs_mfie_mode``);
* plane wave from the observer direction (theta, phi = 0): E_inc = p exp(j k r_o . r),
  p = theta_hat (VV) or phi_hat (HH); far field F_p = -(j k eta / 4 pi) int p.J e^{jk r_o.r'};
  sigma = 4 pi |F|^2 (``bor/solver.py:4457-4473``).

Quadrature, as the reference's:
* far element pairs: 3-point Gauss on both elements (``bor/kernels.py:41``), xi by the
  uniform trapezoid rule with n_xi = 32 ceil((1.5 (2 k c + m_max + 2) + 40 c / R0 + 16) / 32)
  points, c = sqrt(rho rho') (exponentially convergent for the periodic integrand; the
  reference's FFT grid converges to the same values);
* near element pairs (``bor/solver.py:1520-1580``): every pair with |e - f| <= 2, and any
  other pair whose segments come within
  max(1.001 * 8 * 2 pi / 8192 * rho_max(e, f), 2 max(L_e, L_f));
  self pairs and adjacent pairs by graded cells (``bor/solver.py:718,773,795``: the unit
  square split recursively toward the singular set -- the diagonal, or the shared corner --
  to depth 4, each cell a tensor rule of 4 x 5 Gauss points); the other near pairs by a
  12 x 12 Gauss tensor rule (``bor/solver.py:843``);
* near pairs' xi integrals: this restatement's own rule on [0, pi] (using the parity of
  each integrand), converged far below the reference's 2e-8 agreement test
  (``bor/kernels.py:18``): a 20-point sinh-mapped Gauss core xi = delta sinh(v) on [0, a]
  (delta = R0 / c, a = min(4 delta, Delta, pi)), then 16-point Gauss panels
  [a 2^g, a 2^(g+1)] while a 2^g < Delta = 4 pi / (n_max + k c + 1) (two periods of the
  fastest oscillation), and panels of length Delta from there up to pi (the last one cut
  at pi).

Parity pinned against the reference's own per-mode matrices and solves
(``tests/golden/ref_bor_modes.npz``, ``tests/golden/ref_bor_sphere.npz``).
"""
from __future__ import annotations

import math

import numpy as np
from scipy import special as sp

ETA0 = 376.730313668
C0 = 299_792_458.0
FAR_ORDER = 3
CELL_ORDER = 4
CELL_DEPTH = 4
REGULAR_ORDER = 12
NEAR_SPAN = 2
DIRECT_SCALE = 1.001 * 8.0 * 2.0 * math.pi / 8192
XI_CORE = 20
XI_PANEL = 16


def gl(q):
    return np.polynomial.legendre.leggauss(q)


def unit_gl(q):
    x, w = gl(q)
    return 0.5 * (x + 1.0), 0.5 * w


class Body:
    """Generatrix geometry, Gauss points and tents."""

    def __init__(self, points):
        p = np.asarray(points, dtype=np.float64)
        self.nodes = p
        self.ne = len(p) - 1
        self.nn = len(p)
        d = p[1:] - p[:-1]
        self.L = np.hypot(d[:, 0], d[:, 1])
        self.trho = d[:, 0] / self.L
        self.tz = d[:, 1] / self.L
        rmax = max(1.0, float(np.max(p[:, 0])))
        self.on_axis = np.array([p[i, 0] <= 1e-12 * rmax for i in range(self.nn)])

    def points(self, e, s, w):
        """Points on element(s) e at local parameters s in [0,1] with weights w (sum = 1);
        e may be an array matching s."""
        p0, p1 = self.nodes[e], self.nodes[np.asarray(e) + 1]
        rho = p0[..., 0] + s * (p1[..., 0] - p0[..., 0])
        z = p0[..., 1] + s * (p1[..., 1] - p0[..., 1])
        L = self.L[e]
        T0, T1 = 1.0 - s, s
        drho = self.trho[e]
        # d(rho T)/dt = rho dT/dt + T drho/dt
        D0 = rho * (-1.0 / L) + T0 * drho
        D1 = rho * (1.0 / L) + T1 * drho
        return dict(rho=rho, z=z, w=w * L, T=(T0, T1), D=(D0, D1), trho=drho, tz=self.tz[e])

    def pair_classes(self):
        """(ne, ne) uint8: 0 far, 1 self or adjacent (graded cells), 2 other near pairs
        (12 x 12 Gauss), by the reference's near-pair routing."""
        ne = self.ne
        cls = np.zeros((ne, ne), dtype=np.uint8)
        e = np.arange(ne)
        gap = np.abs(e[:, None] - e[None, :])
        cls[gap <= NEAR_SPAN] = 2
        cls[gap <= 1] = 1
        rho_e = np.maximum(self.nodes[:-1, 0], self.nodes[1:, 0])
        pair_gap = np.maximum(DIRECT_SCALE * np.maximum(rho_e[:, None], rho_e[None, :]),
                              2.0 * np.maximum(self.L[:, None], self.L[None, :]))
        a, b = self.nodes[:-1], self.nodes[1:]
        dist = np.minimum(np.minimum(point_segment(a[:, None], a[None, :], b[None, :]),
                                     point_segment(b[:, None], a[None, :], b[None, :])),
                          np.minimum(point_segment(a[None, :], a[:, None], b[:, None]),
                                     point_segment(b[None, :], a[:, None], b[:, None])))
        cls[(gap > NEAR_SPAN) & (dist <= pair_gap)] = 2
        return cls


def point_segment(c, a, b):
    """Distance from points c to segments [a, b] (arrays [..., 2], broadcast)."""
    ab = b - a
    t = np.sum((c - a) * ab, axis=-1) / np.maximum(np.sum(ab * ab, axis=-1), 1e-300)
    t = np.clip(t, 0.0, 1.0)[..., None]
    d = c - (a + t * ab)
    return np.hypot(d[..., 0], d[..., 1])


def far_rule():
    return unit_gl(FAR_ORDER)


def graded_cells(kind, depth=CELL_DEPTH):
    """Cells (s0, s1, p0, p1) of [0,1]^2 refined toward the singular set: 'diag' (s = s'),
    or 'cornerAB' (s = A, s' = B)."""
    out = []

    def touches(s0, s1, p0, p1):
        if kind == 'diag':
            return not (s1 <= p0 or p1 <= s0)
        a, b = float(kind[6]), float(kind[7])
        return s0 <= a <= s1 and p0 <= b <= p1

    def split(s0, s1, p0, p1, d):
        if d >= depth or not touches(s0, s1, p0, p1):
            out.append((s0, s1, p0, p1))
            return
        sm, pm = 0.5 * (s0 + s1), 0.5 * (p0 + p1)
        split(s0, sm, p0, pm, d + 1)
        split(s0, sm, pm, p1, d + 1)
        split(sm, s1, p0, pm, d + 1)
        split(sm, s1, pm, p1, d + 1)

    split(0.0, 1.0, 0.0, 1.0, 0)
    return out


def cell_points(kind, order=CELL_ORDER, depth=CELL_DEPTH):
    """(s, s', w) of the graded-cell rule: per cell order x (order + 1) Gauss points."""
    u, wu = unit_gl(order)
    v, wv = unit_gl(order + 1)
    S, P, W = [], [], []
    for s0, s1, p0, p1 in graded_cells(kind, depth):
        hs, hp = s1 - s0, p1 - p0
        a, b = np.meshgrid(s0 + u * hs, p0 + v * hp, indexing='ij')
        S.append(a.ravel())
        P.append(b.ravel())
        W.append(np.outer(wu * hs, wv * hp).ravel())
    return np.concatenate(S), np.concatenate(P), np.concatenate(W)


def regular_points(order=REGULAR_ORDER):
    u, w = unit_gl(order)
    a, b = np.meshgrid(u, u, indexing='ij')
    return a.ravel(), b.ravel(), np.outer(w, w).ravel()


def pair_rule(e, f, cls):
    """(s, s', w) point pairs of a near element pair."""
    if cls == 1:
        if e == f:
            return cell_points('diag')
        return cell_points('corner10' if f == e + 1 else 'corner01')
    return regular_points()


def n_xi(k, rho_p, rho_q, r0, mmax):
    c = np.sqrt(rho_p * rho_q)
    v = 1.5 * (2.0 * k * c + mmax + 2) + 40.0 * c / np.maximum(r0, 1e-300) + 16.0
    return (32 * np.ceil(v / 32.0)).astype(np.int64)


def near_xi_rule(delta, nmax, kc):
    """Nodes and weights [P, n] on [0, pi] for near pairs (delta = R0 / c per pair, kc =
    k c per pair), grouped: returns a list of (pair indices, xi, w) with one node count
    per group."""
    delta = np.atleast_1d(np.asarray(delta, dtype=np.float64))
    kc = np.broadcast_to(np.asarray(kc, dtype=np.float64), delta.shape)
    span = 4.0 * math.pi / (nmax + kc + 1.0)
    a = np.minimum(np.minimum(4.0 * delta, span), math.pi)
    # panel ends: a 2^g while below span (lengths doubling), then a 2^G + u span, up to pi
    geo = np.zeros(delta.shape, dtype=np.int64)
    while np.any((a * 2.0 ** geo < span) & (a * 2.0 ** geo < math.pi)):
        geo += (a * 2.0 ** geo < span) & (a * 2.0 ** geo < math.pi)
    top = a * 2.0 ** geo
    uni = np.where(top < math.pi, np.ceil((math.pi - top) / span), 0).astype(np.int64)
    uni = np.where(top + (uni - 1) * span >= math.pi, uni - 1, uni)
    width = int(np.max(geo + uni)) + 1
    j = np.arange(width)[None, :]
    ends = np.where(j <= geo[:, None], a[:, None] * 2.0 ** np.minimum(j, geo[:, None]),
                    top[:, None] + (j - geo[:, None]) * span[:, None])
    ends = np.minimum(ends, math.pi)
    ends[j > (geo + uni)[:, None]] = math.pi
    count = np.sum(ends[:, 1:] > ends[:, :-1], axis=1)
    u, wu = unit_gl(XI_CORE)
    g, wg = unit_gl(XI_PANEL)
    out = []
    for c in np.unique(count):
        sel = np.nonzero(count == c)[0]
        d, vmax = delta[sel, None], np.arcsinh(a[sel] / delta[sel])[:, None]
        v = u[None, :] * vmax
        xi = [d * np.sinh(v)]
        w = [d * np.cosh(v) * wu[None, :] * vmax]
        for j in range(c):
            lo, hi = ends[sel, j, None], ends[sel, j + 1, None]
            xi.append(lo + (hi - lo) * g[None, :])
            w.append((hi - lo) * wg[None, :])
        out.append((sel, np.concatenate(xi, axis=1), np.concatenate(w, axis=1)))
    return out


def green(k, rp, zp, rq, zq, xi):
    """e^{-jkR}/(4 pi R) at xi (arrays broadcast)."""
    s = np.sin(0.5 * xi)
    R = np.sqrt((rp - rq) ** 2 + (zp - zq) ** 2 + 4.0 * rp * rq * s * s)
    return np.exp(-1j * k * R) / (4.0 * np.pi * R)


def brackets(k, rp, zp, trp, tzp, rq, zq, trq, tzq, xi):
    """The four MFIE brackets (tt, tf, ft, ff) at xi, cancellation-free form."""
    h = 2.0 * np.sin(0.5 * xi) ** 2
    sx = np.sin(xi)
    dr, dz = rp - rq, zp - zq
    R = np.sqrt(dr * dr + dz * dz + 2.0 * rp * rq * h)
    p = (1.0 + 1j * k * R) * np.exp(-1j * k * R) / (4.0 * np.pi * R ** 3)
    X = trp * tzq - tzp * trq
    D = trp * trq + tzp * tzq
    A = trp * dr + tzp * dz
    N = -tzp * dr + trp * dz
    tt = (A * X - D * N) + h * (A * tzp * trq + trp * rq * X + D * tzp * rq + trp * trq * N)
    tf = -sx * dz * (trp * trp + tzp * tzp)
    ft = sx * (rq * X + trq * N)
    ff = -tzp * rq * h - N * (1.0 - h)
    return -p * tt, -p * tf, -p * ft, -p * ff


def modal_far(k, rp, zp, trp, tzp, rq, zq, trq, tzq, mmax, mfie):
    """Far point pairs: G_n, n = 0..mmax+1 ([P, mmax+2]) and, with mfie, the brackets'
    K_n, n = 0..mmax ([4, P, mmax+1]), by the trapezoid rule."""
    r0 = np.hypot(rp - rq, zp - zq)
    nx = n_xi(k, rp, rq, r0, mmax)
    G = np.zeros((len(rp), mmax + 2), dtype=np.complex128)
    K = np.zeros((4, len(rp), mmax + 1), dtype=np.complex128) if mfie else None
    for n in np.unique(nx):
        sel = np.nonzero(nx == n)[0]
        xi = 2.0 * np.pi * np.arange(n) / n
        d = 2.0 * np.pi / n
        col = lambda a: a[sel, None]
        g = green(k, col(rp), col(zp), col(rq), col(zq), xi[None, :]) * d
        G[sel] = g @ np.cos(np.outer(xi, np.arange(mmax + 2)))
        if mfie:
            F = brackets(k, col(rp), col(zp), col(trp), col(tzp), col(rq), col(zq), col(trq), col(tzq), xi[None, :])
            cm = np.cos(np.outer(xi, np.arange(mmax + 1)))
            sm = np.sin(np.outer(xi, np.arange(mmax + 1)))
            K[0, sel] = (F[0] * d) @ cm
            K[1, sel] = -1j * ((F[1] * d) @ sm)
            K[2, sel] = -1j * ((F[2] * d) @ sm)
            K[3, sel] = (F[3] * d) @ cm
    return G, K


def modal_near(k, rp, zp, trp, tzp, rq, zq, trq, tzq, mmax, mfie):
    """Near point pairs: the same quantities by the near xi rule (parity on [0, pi])."""
    P = len(rp)
    G = np.zeros((P, mmax + 2), dtype=np.complex128)
    K = np.zeros((4, P, mmax + 1), dtype=np.complex128) if mfie else None
    c = np.sqrt(rp * rq)
    r0 = np.hypot(rp - rq, zp - zq)
    for sel, xi, w in near_xi_rule(r0 / c, mmax + 1, k * c):
        col = lambda a: a[sel, None]
        w2 = 2.0 * w
        g = green(k, col(rp), col(zp), col(rq), col(zq), xi) * w2
        if mfie:
            F = [f * w2 for f in brackets(k, col(rp), col(zp), col(trp), col(tzp), col(rq), col(zq), col(trq),
                                          col(tzq), xi)]
        # e^{j n xi} by repeated rotation
        step = np.exp(1j * xi)
        rot = np.ones_like(step)
        for n in range(mmax + 2):
            G[sel, n] = np.sum(g * rot.real, axis=1)
            if mfie and n <= mmax:
                K[0, sel, n] = np.sum(F[0] * rot.real, axis=1)
                K[1, sel, n] = -1j * np.sum(F[1] * rot.imag, axis=1)
                K[2, sel, n] = -1j * np.sum(F[2] * rot.imag, axis=1)
                K[3, sel, n] = np.sum(F[3] * rot.real, axis=1)
            rot = rot * step
    return G, K


def mode_kernels(G, m):
    """(G_|m|, (G_|m-1| + G_|m+1|)/2, (G_|m-1| - G_|m+1|)/2) from G[..., 0..mmax+1]."""
    a = abs(m)
    g0 = G[..., a]
    gm1 = G[..., abs(m - 1)]
    gp1 = G[..., abs(m + 1)]
    return g0, 0.5 * (gm1 + gp1), 0.5 * (gm1 - gp1)


class Assembler:
    """Point pairs of every element pair with their modal kernels (all modes), and the
    per-mode 2Nn x 2Nn EFIE / MFIE matrices (before the pole reduction)."""

    def __init__(self, body, k, mmax, mfie=False):
        self.b = body
        self.k = float(k)
        self.mmax = int(mmax)
        self.mfie = bool(mfie)
        cls = body.pair_classes()
        s3, w3 = far_rule()
        far = (np.repeat(s3, FAR_ORDER), np.tile(s3, FAR_ORDER), np.repeat(w3, FAR_ORDER) * np.tile(w3, FAR_ORDER))
        E, F, S, Sq, W = [], [], [], [], []
        for e in range(body.ne):
            for f in range(body.ne):
                s, sq, w = far if cls[e, f] == 0 else pair_rule(e, f, cls[e, f])
                E.append(np.full(len(s), e))
                F.append(np.full(len(s), f))
                S.append(s)
                Sq.append(sq)
                W.append(w)
        self.E, self.F = np.concatenate(E), np.concatenate(F)
        self.near = cls[self.E, self.F] > 0
        self.pe = body.points(self.E, np.concatenate(S), np.concatenate(W))
        self.pf = body.points(self.F, np.concatenate(Sq), 1.0)
        P = len(self.E)
        self.G = np.zeros((P, self.mmax + 2), dtype=np.complex128)
        self.K = np.zeros((4, P, self.mmax + 1), dtype=np.complex128) if self.mfie else None
        for sel, fun in ((np.nonzero(~self.near)[0], modal_far), (np.nonzero(self.near)[0], modal_near)):
            if len(sel) == 0:
                continue
            pe, pf = self.pe, self.pf
            G, K = fun(self.k, pe['rho'][sel], pe['z'][sel], pe['trho'][sel], pe['tz'][sel], pf['rho'][sel],
                       pf['z'][sel], pf['trho'][sel], pf['tz'][sel], self.mmax, self.mfie)
            self.G[sel] = G
            if self.mfie:
                self.K[:, sel] = K

    def _scatter(self, Z, ro, co, values):
        """Z[ro + E + a, co + F + c] += sum over point pairs of values[a][c]."""
        for a in range(2):
            for c in range(2):
                np.add.at(Z, (ro + self.E + a, co + self.F + c), values[a][c])

    def matrix(self, m):
        """EFIE matrix of signed mode m."""
        k, nn = self.k, self.b.nn
        pe, pf = self.pe, self.pf
        Z = np.zeros((2 * nn, 2 * nn), dtype=np.complex128)
        g0, gc, gs = mode_kernels(self.G, m)
        ww = pe['w'] * pf['w']
        rr = pe['rho'] * pf['rho'] * ww
        ktt = rr * (pe['trho'] * pf['trho'] * gc + pe['tz'] * pf['tz'] * g0)
        ktf = rr * (-1j * pe['trho']) * gs
        kft = rr * (1j * pf['trho']) * gs
        kff = rr * gc
        ks = ww * g0
        Tp, Dp, Tq, Dq = pe['T'], pe['D'], pf['T'], pf['D']
        r2 = range(2)
        self._scatter(Z, 0, 0, [[Tp[a] * ktt * Tq[c] - Dp[a] * ks * Dq[c] / k ** 2 for c in r2] for a in r2])
        self._scatter(Z, 0, nn, [[Tp[a] * ktf * Tq[c] - (1j * m) * Dp[a] * ks * Tq[c] / k ** 2 for c in r2]
                                 for a in r2])
        self._scatter(Z, nn, 0, [[Tp[a] * kft * Tq[c] + (1j * m) * Tp[a] * ks * Dq[c] / k ** 2 for c in r2]
                                 for a in r2])
        self._scatter(Z, nn, nn, [[Tp[a] * kff * Tq[c] - (m * m) * Tp[a] * ks * Tq[c] / k ** 2 for c in r2]
                                  for a in r2])
        return (1j * k * ETA0 * 2.0 * np.pi) * Z

    def mass(self):
        """M_ij = 2 pi int rho T_i T_j dt (3-point Gauss per element), [Nn, Nn]."""
        b = self.b
        s, w = far_rule()
        M = np.zeros((b.nn, b.nn))
        for e in range(b.ne):
            p = b.points(e, s, w)
            for a in range(2):
                for c in range(2):
                    M[e + a, e + c] += 2.0 * np.pi * np.sum(p['w'] * p['rho'] * p['T'][a] * p['T'][c])
        return M

    def mfie_matrix(self, m):
        """MFIE matrix (1/2) M - K of signed mode m."""
        if not self.mfie:
            raise ValueError('Assembler built without the MFIE brackets')
        nn = self.b.nn
        pe, pf = self.pe, self.pf
        Z = np.zeros((2 * nn, 2 * nn), dtype=np.complex128)
        rr = pe['rho'] * pf['rho'] * pe['w'] * pf['w']
        for uv, (ro, co) in enumerate(((0, 0), (0, nn), (nn, 0), (nn, nn))):
            km = self.K[uv, :, abs(m)] * (-1.0 if (uv in (1, 2) and m < 0) else 1.0)
            self._scatter(Z, ro, co, [[-2.0 * np.pi * pe['T'][a] * rr * km * pf['T'][c] for c in range(2)]
                                      for a in range(2)])
        M = self.mass()
        Z[:nn, :nn] += 0.5 * M
        Z[nn:, nn:] += 0.5 * M
        return Z

    def cfie_matrix(self, m, alpha=0.5):
        return alpha * self.matrix(m) + (1.0 - alpha) * ETA0 * self.mfie_matrix(m)


def pole_transform(body, m):
    """Q (2Nn x n_active): active nodal components; |m| = 1 ties the pole phi to t."""
    nn = body.nn
    t_act = np.ones(nn, dtype=bool)
    f_act = np.ones(nn, dtype=bool)
    for end in (0, nn - 1):
        if body.on_axis[end]:
            t_act[end] = abs(m) == 1
            f_act[end] = False
        else:
            t_act[end] = False
            f_act[end] = True
    act = np.nonzero(np.concatenate([t_act, f_act]))[0]
    Q = np.zeros((2 * nn, len(act)), dtype=np.complex128)
    Q[act, np.arange(len(act))] = 1.0
    if abs(m) == 1:
        for end, el in ((0, 0), (nn - 1, body.ne - 1)):
            if not body.on_axis[end]:
                continue
            col = int(np.nonzero(act == end)[0][0])
            Q[nn + end, col] = 1j * m * (1.0 if body.trho[el] >= 0 else -1.0)
    return Q


def excitation(body, k, thetas_deg, m, far=False, kind='efie'):
    """Columns [VV..., HH...] (2Nn x 2 n_theta) of <W_i, E_inc> (kind 'efie'),
    eta0 <W_i, n x H_inc> (kind 'mfie'), or far-field weights (far=True)."""
    s, w = far_rule()
    nn = body.nn
    th = np.deg2rad(np.asarray(thetas_deg, dtype=np.float64))
    nt = len(th)
    V = np.zeros((2 * nn, 2 * nt), dtype=np.complex128)
    ct, st = np.cos(th), np.sin(th)
    for e in range(body.ne):
        p = body.points(e, s, w)
        x = k * np.outer(p['rho'], st)             # (q, nt)
        ph = np.exp(1j * k * np.outer(p['z'], ct)) * (p['rho'] * p['w'])[:, None]
        jm = sp.jv(m, x)
        jm1 = sp.jv(m - 1, x)
        jp1 = sp.jv(m + 1, x)
        I0 = 2 * np.pi * (1j ** m) * jm
        Ic = np.pi * ((1j ** (m + 1)) * jp1 + (1j ** (m - 1)) * jm1)
        Is = -1j * np.pi * ((1j ** (m - 1)) * jm1 - (1j ** (m + 1)) * jp1)
        if far:
            Is = -Is
        if kind == 'mfie' and not far:
            vt_v = ph * Ic
            vf_v = ph * (-p['trho'] * Is)
            vt_h = ph * (ct[None, :] * Is)
            vf_h = ph * (p['trho'] * ct[None, :] * Ic - p['tz'] * st[None, :] * I0)
        else:
            vt_v = ph * (p['trho'] * ct[None, :] * Ic - p['tz'] * st[None, :] * I0)
            vf_v = ph * (-ct[None, :] * Is)
            vt_h = ph * (p['trho'] * Is)
            vf_h = ph * Ic
        for a in range(2):
            T = p['T'][a][:, None]
            i = e + a
            V[i, :nt] += np.sum(T * vt_v, axis=0)
            V[nn + i, :nt] += np.sum(T * vf_v, axis=0)
            V[i, nt:] += np.sum(T * vt_h, axis=0)
            V[nn + i, nt:] += np.sum(T * vf_h, axis=0)
    return V


def solve(points, k, thetas_deg, mmax, formulation='efie', alpha=0.5):
    """Monostatic VV/HH far-field amplitudes and sigma (m^2) summing modes -mmax..mmax
    (formulation 'efie', 'cfie' with weight alpha, or 'mfie' = alpha 0)."""
    body = Body(points)
    if formulation == 'mfie':
        alpha = 0.0
    cfie = formulation in ('cfie', 'mfie')
    asm = Assembler(body, k, mmax, mfie=cfie)
    nt = len(thetas_deg)
    F = np.zeros(2 * nt, dtype=np.complex128)
    for m in range(-mmax, mmax + 1):
        Z = asm.cfie_matrix(m, alpha) if cfie else asm.matrix(m)
        Q = pole_transform(body, m)
        Zr = Q.conj().T @ Z @ Q
        Vf = excitation(body, k, thetas_deg, m)
        if cfie:
            Vf = alpha * Vf + (1.0 - alpha) * excitation(body, k, thetas_deg, m, kind='mfie')
        V = Q.conj().T @ Vf
        W = Q.T @ excitation(body, k, thetas_deg, m, far=True)
        x = np.linalg.solve(Zr, V)
        F += np.sum(W * x, axis=0)
    F *= -1j * k * ETA0 / (4.0 * np.pi)
    Fv, Fh = F[:nt], F[nt:]
    return dict(amp_vv=Fv, amp_hh=Fh, sigma_vv=4 * np.pi * np.abs(Fv) ** 2, sigma_hh=4 * np.pi * np.abs(Fh) ** 2)
