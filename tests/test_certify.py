"""Mesh-convergence certification (reference runs/quality.py:166-547, twod/solver.py
_certify_2d_results) against the reference's own outputs on the same inputs
(tests/golden/mesh_certification.json, made by tests/golden/make_quality_golden.py)."""
import json
import math
import os

import pytest

from grim_20261007_b200.twod import certify as C

GOLDEN = os.path.join(os.path.dirname(__file__), 'golden', 'mesh_certification.json')


@pytest.fixture(scope='module')
def g():
    with open(GOLDEN) as f:
        return json.load(f)


def test_panel_density_refinement_matches_reference(g):
    for factor, ref in g['scaled'].items():
        assert C.scale_snapshot_panel_density(g['snapshot'], float(factor)) == ref


def test_default_policy_matches_reference(g):
    assert C.validate_policy(None) == g['policy_default']
    with pytest.raises(ValueError):
        C.validate_policy({'fine_factor': 1.0})
    with pytest.raises(ValueError):
        C.validate_policy({'bogus': 1})


@pytest.mark.parametrize('name', ['small', 'large'])
def test_convergence_report_matches_reference(g, name):
    got = C.evaluate_mesh_convergence({'samples': g['base']}, {'samples': g[name]}, 1.0, 3.0)
    ref = g['reports'][name]
    assert set(got) == set(ref)
    for key, val in ref.items():
        if isinstance(val, float):
            assert math.isclose(got[key], val, rel_tol=1e-12, abs_tol=1e-14), key
        elif isinstance(val, dict):
            for k2, v2 in val.items():
                assert math.isclose(got[key][k2], v2, rel_tol=1e-12, abs_tol=1e-14), (key, k2)
        else:
            assert got[key] == val, key


def test_certify_publishes_fine_or_raises(g):
    policy = C.validate_policy(None)
    base = {'samples': g['base'], 'metadata': {'quality_gate': {'passed': True}}}
    fine = {'samples': g['small'], 'metadata': {'quality_gate': {'passed': True}}}
    out = C.certify(base, fine, policy, 100, 150)
    assert out['samples'] is g['small'] and out['metadata']['mesh_convergence_certified']
    assert out['metadata']['mesh_convergence']['panel_refinement_ratio'] == 1.5
    with pytest.raises(ValueError, match='convergence failed'):
        C.certify(base, {'samples': g['large'], 'metadata': {}}, policy, 100, 150)
    with pytest.raises(ValueError, match='refinement failed'):
        C.certify(base, fine, policy, 100, 100)
