"""FP64 oracle: body-of-revolution PEC EFIE per azimuthal mode (test infrastructure).

Restates the physics of the reference's BoR solver (``ghost_backend/bor``):

* generatrix (rho, z) polyline from the +z pole to the -z pole
  (``bor/kernels.py:63`` ``Generatrix``); 3 Gauss points per element for far pairs
  (``bor/kernels.py:41`` ``FAR_GAUSS_ORDER``);
* unknowns: nodal tents T_i(t) for the t- and phi-directed surface current,
  J = sum_m e^{j m phi} sum_i (a_i T_i t_hat + b_i T_i phi_hat)  (n_dofs = 2 Nn,
  ``bor/solver.py:4160``);
* axis poles: the phi component is inactive and the t component is active only for
  |m| = 1, where it is tied to phi by J_phi = j m sign(t_rho) J_t
  (``bor/solver.py:2369-2440`` ``basis_mask`` / ``basis_transform``, Galerkin
  reduction Q^H Z Q);
* Galerkin EFIE, time convention e^{+j w t}:
  Z = j k eta 2 pi [ <W.J> - (1/k^2) <div W, div J> ] with the modal Green's function
  G_m = int_0^{2 pi} e^{-jkR}/(4 pi R) cos(m xi) d xi,
  R^2 = (rho - rho')^2 + (z - z')^2 + 4 rho rho' sin^2(xi/2)
  (``bor/solver.py:1769-1827`` ``assemble_mode``, ``bor/bor_stream_kernel.c:48``);
* plane wave from the observer direction (theta, phi = 0): E_inc = p exp(j k r_o . r),
  p = theta_hat (VV) or phi_hat (HH); far field F_p = -(j k eta / 4 pi) int p.J e^{jk r_o.r'};
  sigma = 4 pi |F|^2 (``bor/solver.py:4457-4473``).

Quadrature (this restatement's own rules; the GPU path uses the same ones):
* far element pairs: 3-point Gauss on both elements, xi by the uniform trapezoid rule
  with n_xi = 32 ceil((1.5 (2 k sqrt(rho rho') + m_max + 2) + 30 sqrt(rho rho')/R0 + 16) / 32)
  points (exponentially convergent for the periodic integrand);
* near pairs (same or adjacent element): the source element is split at the point
  nearest the observation point and each piece integrated by a cubically graded
  8-point Gauss rule; xi by a 32-point Gauss rule after the sinh substitution
  xi = (R0/c) sinh(u), c = sqrt(rho rho') (Johnston & Elliott, 2005), which removes the
  near-singularity of 1/R at xi = 0.
"""
from __future__ import annotations

import math

import numpy as np
from scipy import special as sp

ETA0 = 376.730313668
C0 = 299_792_458.0
FAR_ORDER = 3
NEAR_ORDER = 8
NEAR_XI_ORDER = 32


def gl(q):
    return np.polynomial.legendre.leggauss(q)


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
        """Points on element e at local parameters s in [0,1] with weights w (sum = 1)."""
        p0, p1 = self.nodes[e], self.nodes[e + 1]
        rho = p0[0] + s * (p1[0] - p0[0])
        z = p0[1] + s * (p1[1] - p0[1])
        L = self.L[e]
        T0, T1 = 1.0 - s, s
        drho = self.trho[e]
        # d(rho T)/dt = rho dT/dt + T drho/dt
        D0 = rho * (-1.0 / L) + T0 * drho
        D1 = rho * (1.0 / L) + T1 * drho
        return dict(rho=rho, z=z, w=w * L, T=(T0, T1), D=(D0, D1), trho=drho, tz=self.tz[e])


def far_rule():
    x, w = gl(FAR_ORDER)
    return 0.5 * (x + 1.0), 0.5 * w


def graded_rule(a, b, toward, q=NEAR_ORDER):
    """Cubically graded Gauss rule on [a, b] clustered at ``toward`` (a or b)."""
    x, w = gl(q)
    u = 0.5 * (x + 1.0)
    wu = 0.5 * w
    if toward == a:
        s = a + (b - a) * u ** 3
        ws = (b - a) * 3 * u ** 2 * wu
    else:
        s = b - (b - a) * u ** 3
        ws = (b - a) * 3 * u ** 2 * wu
    return s, ws


def n_xi(k, rho_p, rho_q, r0, mmax):
    c = np.sqrt(rho_p * rho_q)
    v = 1.5 * (2.0 * k * c + mmax + 2) + 30.0 * c / np.maximum(r0, 1e-300) + 16.0
    return (32 * np.ceil(v / 32.0)).astype(np.int64)


def modal_trapezoid(k, rp, zp, rq, zq, mmax):
    """G_m, m = 0..mmax+1, by the uniform trapezoid rule (vectorised over pairs)."""
    rp, zp, rq, zq = map(np.atleast_1d, (rp, zp, rq, zq))
    r0 = np.hypot(rp - rq, zp - zq)
    nx = n_xi(k, rp, rq, r0, mmax)
    out = np.zeros((len(rp), mmax + 2), dtype=np.complex128)
    m = np.arange(mmax + 2)
    for n in np.unique(nx):
        sel = np.nonzero(nx == n)[0]
        xi = 2.0 * np.pi * np.arange(n) / n
        s2 = np.sin(0.5 * xi) ** 2
        R = np.sqrt(r0[sel, None] ** 2 + 4.0 * rp[sel, None] * rq[sel, None] * s2[None, :])
        g = np.exp(-1j * k * R) / (4.0 * np.pi * R) * (2.0 * np.pi / n)
        out[sel] = g @ np.cos(np.outer(xi, m))
    return out


def modal_sinh(k, rp, zp, rq, zq, mmax, q=NEAR_XI_ORDER):
    """G_m by the sinh-substituted Gauss rule on xi in [-pi, pi] (near pairs)."""
    rp, zp, rq, zq = map(np.atleast_1d, (rp, zp, rq, zq))
    r0 = np.maximum(np.hypot(rp - rq, zp - zq), 1e-300)
    c = np.sqrt(rp * rq)
    x, w = gl(q)
    umax = np.arcsinh(c * np.pi / r0)
    u = x[None, :] * umax[:, None]
    wu = w[None, :] * umax[:, None]
    xi = (r0 / c)[:, None] * np.sinh(u)
    dxi = (r0 / c)[:, None] * np.cosh(u) * wu
    R = np.sqrt(r0[:, None] ** 2 + 4.0 * (rp * rq)[:, None] * np.sin(0.5 * xi) ** 2)
    g = np.exp(-1j * k * R) / (4.0 * np.pi * R) * dxi
    m = np.arange(mmax + 2)
    return np.einsum('pq,pqm->pm', g, np.cos(xi[:, :, None] * m[None, None, :]))


def mode_kernels(G, m):
    """(G_|m|, (G_|m-1| + G_|m+1|)/2, (G_|m-1| - G_|m+1|)/2) from G[..., 0..mmax+1]."""
    a = abs(m)
    g0 = G[..., a]
    gm1 = G[..., abs(m - 1)]
    gp1 = G[..., abs(m + 1)]
    return g0, 0.5 * (gm1 + gp1), 0.5 * (gm1 - gp1)


class Assembler:
    """Element-pair modal kernels (all modes) and per-mode 2Nn x 2Nn EFIE matrices."""

    def __init__(self, body, k, mmax):
        self.b = body
        self.k = float(k)
        self.mmax = int(mmax)
        s, w = far_rule()
        self.far = [body.points(e, s, w) for e in range(body.ne)]
        self.pairs = []  # (e, f, obs pts dict, src pts dict, G[Pe, Pf, mmax+2])
        for e in range(body.ne):
            pe = self.far[e]
            for f in range(body.ne):
                if abs(e - f) <= 1:
                    self._near_pair(e, f)
                else:
                    pf = self.far[f]
                    rp = np.repeat(pe['rho'], FAR_ORDER)
                    zp = np.repeat(pe['z'], FAR_ORDER)
                    rq = np.tile(pf['rho'], FAR_ORDER)
                    zq = np.tile(pf['z'], FAR_ORDER)
                    G = modal_trapezoid(self.k, rp, zp, rq, zq, self.mmax)
                    self.pairs.append((e, f, pe, pf, G.reshape(FAR_ORDER, FAR_ORDER, -1)))

    def _near_pair(self, e, f):
        b = self.b
        pe = self.far[e]
        for ip in range(FAR_ORDER):
            # source rule on f, graded toward the point of f nearest to obs point ip
            if e == f:
                sp_ = float(pe_s(ip))
                s1, w1 = graded_rule(0.0, sp_, sp_)
                s2, w2 = graded_rule(sp_, 1.0, sp_)
                s, w = np.concatenate([s1, s2]), np.concatenate([w1, w2])
            elif f == e + 1:
                s, w = graded_rule(0.0, 1.0, 0.0)
            else:
                s, w = graded_rule(0.0, 1.0, 1.0)
            pf = b.points(f, s, w)
            one = {kk: (v[ip:ip + 1] if isinstance(v, np.ndarray) else v) for kk, v in pe.items() if kk not in ('T', 'D')}
            one['T'] = (pe['T'][0][ip:ip + 1], pe['T'][1][ip:ip + 1])
            one['D'] = (pe['D'][0][ip:ip + 1], pe['D'][1][ip:ip + 1])
            n = len(s)
            G = modal_sinh(self.k, np.full(n, pe['rho'][ip]), np.full(n, pe['z'][ip]), pf['rho'], pf['z'], self.mmax)
            self.pairs.append((e, f, one, pf, G.reshape(1, n, -1)))

    def matrix(self, m):
        """Full 2Nn x 2Nn EFIE matrix of signed mode m (before the pole reduction)."""
        b, k = self.b, self.k
        nn = b.nn
        Z = np.zeros((2 * nn, 2 * nn), dtype=np.complex128)
        for e, f, pe, pf, G in self.pairs:
            g0, gc, gs = mode_kernels(G, m)
            rr = np.outer(pe['rho'] * pe['w'], pf['rho'] * pf['w'])
            ww = np.outer(pe['w'], pf['w'])
            ktt = rr * (pe['trho'] * pf['trho'] * gc + pe['tz'] * pf['tz'] * g0)
            ktf = rr * (-1j * pe['trho']) * gs
            kft = rr * (1j * pf['trho']) * gs
            kff = rr * gc
            ks = ww * g0
            for a in range(2):
                Ta, Da = pe['T'][a], pe['D'][a]
                i = e + a
                for c in range(2):
                    Tc, Dc = pf['T'][c], pf['D'][c]
                    jn = f + c
                    Z[i, jn] += Ta @ ktt @ Tc - (Da @ ks @ Dc) / k ** 2
                    Z[i, nn + jn] += Ta @ ktf @ Tc - (1j * m) * (Da @ ks @ Tc) / k ** 2
                    Z[nn + i, jn] += Ta @ kft @ Tc + (1j * m) * (Ta @ ks @ Dc) / k ** 2
                    Z[nn + i, nn + jn] += Ta @ kff @ Tc - (m * m) * (Ta @ ks @ Tc) / k ** 2
        return (1j * k * ETA0 * 2.0 * np.pi) * Z


def pe_s(ip):
    s, _ = far_rule()
    return s[ip]


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


def excitation(body, k, thetas_deg, m, far=False):
    """Columns [VV..., HH...] (2Nn x 2 n_theta) of <W_i, E_inc> (far=True: far-field weights)."""
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


def solve(points, k, thetas_deg, mmax):
    """Monostatic VV/HH far-field amplitudes and sigma (m^2) summing modes -mmax..mmax."""
    body = Body(points)
    asm = Assembler(body, k, mmax)
    nt = len(thetas_deg)
    F = np.zeros(2 * nt, dtype=np.complex128)
    for m in range(-mmax, mmax + 1):
        Z = asm.matrix(m)
        Q = pole_transform(body, m)
        Zr = Q.conj().T @ Z @ Q
        V = Q.conj().T @ excitation(body, k, thetas_deg, m)
        W = Q.T @ excitation(body, k, thetas_deg, m, far=True)
        x = np.linalg.solve(Zr, V)
        F += np.sum(W * x, axis=0)
    F *= -1j * k * ETA0 / (4.0 * np.pi)
    Fv, Fh = F[:nt], F[nt:]
    return dict(amp_vv=Fv, amp_hh=Fh, sigma_vv=4 * np.pi * np.abs(Fv) ** 2, sigma_hh=4 * np.pi * np.abs(Fh) ** 2)
