"""Analytic PEC cylinder and sphere backscatter (test infrastructure).

Restated from the reference's validation oracles:

* ``ghost_backend/validation/cylinder.py:37-72``: the complex 2-D backscatter
  amplitude in the solver convention B = -4j sum_n a_n (-1)^n with
  TM a_n = -J_n(ka)/H_n^(2)(ka) and TE a_n = -J_n'(ka)/H_n^(2)'(ka), truncated at
  N = max(10, ceil(ka + 4.05 ka^(1/3) + 2) + 10); sigma_2D = |B|^2 / (4k).
* ``ghost_backend/validation/sphere.py:196`` (``sigma_pec_sphere``): monostatic
  radar cross-section of a PEC sphere from the Mie coefficients
  a_n = psi_n(x)/xi_n(x)-type ratios; here written with the classical backscatter
  sum sigma = (lambda^2 / (4 pi)) |sum_n (-1)^n (2n+1)(a_n - b_n)|^2
  (Bohren & Huffman eq. 4.53 specialised to a perfect conductor).

Pinned against the reference functions' own outputs in ``tests/golden/mie_*.npz``.
"""
from __future__ import annotations

import math

import numpy as np
from scipy import special as sp

C0 = 299_792_458.0


def _nmax_cylinder(ka, pad=10):
    ka = abs(complex(ka))
    return max(10, int(np.ceil(ka + 4.05 * ka ** (1.0 / 3.0) + 2.0)) + pad)


def cylinder_amplitude(radius_m, k, polarization):
    """Stored-convention complex backscatter amplitude B of a PEC circular cylinder."""
    ka = k * radius_m
    n = np.arange(-_nmax_cylinder(ka), _nmax_cylinder(ka) + 1)
    if polarization.upper() == 'TM':
        a = -sp.jv(n, ka) / sp.hankel2(n, ka)
    else:
        a = -sp.jvp(n, ka, 1) / sp.h2vp(n, ka, 1)
    return complex(-4.0j * np.sum(a * (-1.0) ** n))


def cylinder_sigma(radius_m, k, polarization):
    return abs(cylinder_amplitude(radius_m, k, polarization)) ** 2 / (4.0 * k)


def _nmax_sphere(x, pad=12):
    x = abs(x)
    return max(6, int(math.ceil(x + 4.05 * x ** (1.0 / 3.0))) + pad)


def sphere_sigma(radius_m, k):
    """Monostatic RCS (m^2) of a PEC sphere."""
    x = k * radius_m
    nmax = _nmax_sphere(x)
    n = np.arange(1, nmax + 1)
    # Riccati-Bessel psi_n = x j_n(x), xi_n = x h_n^(2)(x), derivatives by recurrence.
    jn = sp.spherical_jn(n, x)
    jnm1 = sp.spherical_jn(n - 1, x)
    yn = sp.spherical_yn(n, x)
    ynm1 = sp.spherical_yn(n - 1, x)
    psi = x * jn
    dpsi = x * jnm1 - n * jn
    xi = x * (jn - 1j * yn)
    dxi = x * (jnm1 - 1j * ynm1) - n * (jn - 1j * yn)
    a = dpsi / dxi
    b = psi / xi
    s = np.sum((-1.0) ** n * (2 * n + 1) * (a - b))
    lam = 2.0 * math.pi / k
    return float(lam ** 2 / (4.0 * math.pi) * abs(s) ** 2)
