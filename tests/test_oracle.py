"""The FP64 oracle pinned against the reference's own outputs (tests/golden/*.npz)."""
import math
import os

import numpy as np
import pytest
from scipy import integrate, special as sp

from oracle import mie, pulse2d as P
from grim_20261007_b200 import synthetic as S
from tests.conftest import GOLDEN


def _golden(name):
    return np.load(os.path.join(GOLDEN, name))


def test_mie_cylinder_matches_reference_validation():
    g = _golden('mie_cylinder.npz')
    for p, pol in enumerate(('TM', 'TE')):
        for i, ka in enumerate(g['ka']):
            a = mie.cylinder_amplitude(1.0, float(ka), pol)
            assert abs(a - g['amplitude'][p, i]) <= 1e-13 * abs(g['amplitude'][p, i])
            assert math.isclose(mie.cylinder_sigma(1.0, float(ka), pol), g['sigma'][p, i], rel_tol=1e-12)


def test_mie_sphere_matches_reference_validation():
    g = _golden('mie_sphere.npz')
    for i, ka in enumerate(g['ka']):
        assert math.isclose(mie.sphere_sigma(1.0, float(ka)), g['sigma'][i], rel_tol=1e-12)


def test_tm_self_term_series_matches_quadrature():
    for k, h in ((10.0, 0.0157), (630.0, 0.0025), (3.0, 1.2)):
        ref_re = integrate.quad(lambda t: 0.25 * sp.y0(k * t), 0, h, limit=200, points=[0.0])[0] * 2
        ref_im = integrate.quad(lambda t: 0.25 * sp.j0(k * t), 0, h, limit=200)[0] * 2
        got = P.tm_self_term(k, h)
        assert abs(got - complex(ref_re, ref_im)) <= 1e-10 * abs(complex(ref_re, ref_im))


def test_pulse_tm_matches_reference_solver_c1():
    """Reference solver (linear Galerkin S+gamma D) vs pulse EFIE on the same 200-gon, 360 angles."""
    g = _golden('ref_cylinder_c1.npz')
    v = S.circle(1.0, 200)
    out = P.solve(float(g['k']), [v], g['angles'], 'TM')
    db = 10 * np.log10(out['sigma'] / g['sigma_TM'])
    assert np.max(np.abs(db)) < 1e-3
    rel = np.abs(out['amplitude'] - g['amp_TM']) / np.abs(g['amp_TM'])
    assert np.max(rel) < 1e-3


def test_pulse_te_matches_reference_solver_c1():
    g = _golden('ref_cylinder_c1.npz')
    v = S.circle(1.0, 200)
    out = P.solve(float(g['k']), [v], g['angles'], 'TE')
    db = 10 * np.log10(out['sigma'] / g['sigma_TE'])
    assert np.max(np.abs(db)) < 0.05


@pytest.mark.parametrize('pol,tol_db', [('TM', 1e-3), ('TE', 0.05)])
def test_pulse_against_mie(pol, tol_db):
    k = 10.0
    out = P.solve(k, [S.circle(1.0, 200)], [0.0], pol)
    ref = mie.cylinder_sigma(1.0, k, pol)
    assert abs(10 * np.log10(out['sigma'][0] / ref)) < tol_db


def test_oracle_backward_error_and_monostatic_symmetry():
    k = 10.0
    out = P.solve(k, [S.circle(1.0, 96)], [0.0, 90.0, 180.0, 270.0], 'TM')
    be = P.backward_error(out['matrix'], out['density'], out['rhs'])
    assert np.max(be) < 1e-14
    # a regular polygon with 4-fold symmetric vertex set: identical sigma at 0/90/180/270
    assert np.ptp(out['sigma']) < 1e-9 * out['sigma'][0]


def test_gauss_rules_and_quadrature_orders():
    delta = np.array([0.5, 1.99, 2.0, 5.99, 6.0, 100.0])
    assert P.quad_order(delta).tolist() == [12, 12, 6, 6, 4, 4]
    for q in (4, 6, 12):
        x, w = P.gauss_legendre(q)
        assert abs(np.sum(w) - 2.0) < 1e-14
        assert abs(np.sum(w * x ** 2) - 2.0 / 3.0) < 1e-14
