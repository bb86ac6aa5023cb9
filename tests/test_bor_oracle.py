"""The body-of-revolution oracle against the reference's own per-mode operators and solves
(tests/golden/ref_bor_modes.npz, made by tests/golden/make_bor_golden.py)."""
import os

import numpy as np
import pytest

from oracle import bor as OB
from tests.conftest import GOLDEN

G = np.load(os.path.join(GOLDEN, 'ref_bor_modes.npz'))


@pytest.fixture(scope='module', params=['sphere', 'graded'])
def body_case(request):
    name = request.param
    body = OB.Body(G[f'{name}_points'])
    asm = OB.Assembler(body, float(G[f'{name}_k']), int(G[f'{name}_mmax']), mfie=True)
    return name, body, asm


def test_near_pair_routing_includes_gap_pairs(body_case):
    name, body, _asm = body_case
    cls = body.pair_classes()
    e = np.arange(body.ne)
    far_apart = np.abs(e[:, None] - e[None, :]) > 2
    if name == 'graded':
        assert np.any((cls == 2) & far_apart)  # short pole elements reach past the span
    assert np.all(cls[~far_apart] > 0)


@pytest.mark.parametrize('m', [0, 1, -1, 2, -3])
def test_mode_operators_match_reference(body_case, m):
    """EFIE and MFIE node matrices: near pairs (graded cells, 12 x 12 Gauss) and far pairs
    equal the reference's to rounding."""
    name, _body, asm = body_case
    for kind, ours in (('efie', asm.matrix(m)), ('mfie', asm.mfie_matrix(m))):
        ref = G[f'{name}_{kind}_{m}']
        assert np.max(np.abs(ours - ref)) <= 1e-13 * np.max(np.abs(ref)), kind


@pytest.mark.parametrize('m', [0, 1, -1, 2, -3])
def test_excitations_match_reference(body_case, m):
    name, body, asm = body_case
    angles = G['angles']
    n = len(angles)
    for kind, tag, scale in (('efie', 'rhs', 1.0), ('mfie', 'rhs_mfie', OB.ETA0)):
        ours = OB.excitation(body, asm.k, angles, m, kind=kind)
        ref = G[f'{name}_{tag}_{m}'] * scale  # [pol, dof, angle]
        for p in range(2):
            got = ours[:, p * n:(p + 1) * n]
            assert np.max(np.abs(got - ref[p])) <= 1e-12 * max(np.max(np.abs(ref[p])), 1e-300), (kind, p)


def test_cfie_solve_matches_reference_sphere():
    """The reference's CFIE far field of the 45-element sphere at ka = 3 (its adaptive
    mode count)."""
    k = 2.0 * np.pi * float(G['sphere45_freq_hz']) / OB.C0
    o = OB.solve(G['sphere45_points'], k, G['sphere45_thetas'], int(G['sphere45_modes_used']), formulation='cfie')
    for pol in ('vv', 'hh'):
        ref = G[f'sphere45_amp_{pol}']
        assert np.max(np.abs(o[f'amp_{pol}'] - ref)) <= 1e-8 * np.max(np.abs(ref))


def test_resonant_sphere_efie_and_cfie_match_reference():
    """Next to the sphere's first interior resonance the EFIE and the CFIE differ; each
    matches the reference's own solve, and the CFIE stays on the Mie value."""
    pts = G['resonant_points']
    k = 2.0 * np.pi * float(G['resonant_freq_hz']) / OB.C0
    th = G['resonant_thetas']
    for form in ('efie', 'cfie'):
        o = OB.solve(pts, k, th, 12, formulation=form)
        for pol in ('vv', 'hh'):
            ref = G[f'resonant_{form}_amp_{pol}']
            assert np.max(np.abs(o[f'amp_{pol}'] - ref)) <= 1e-8 * np.max(np.abs(ref)), (form, pol)
    mie_db = 10 * np.log10(float(G['resonant_mie_sigma']))
    cfie_db = 10 * np.log10(4 * np.pi * np.abs(G['resonant_cfie_amp_vv'][0]) ** 2)
    assert abs(cfie_db - mie_db) < 0.05
