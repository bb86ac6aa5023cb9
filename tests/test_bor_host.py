"""BoR host logic (no GPU): pole reduction map, mode limits, sample counts."""
import os

import numpy as np
import pytest

from grim_20261007_b200 import synthetic as S
from grim_20261007_b200.bor import solver as B
from oracle import bor as OB
from tests.conftest import GOLDEN


def _q_from_map(rf, rw, nred, nn):
    Q = np.zeros((2 * nn, nred), dtype=complex)
    for r in range(nred):
        for i in range(2):
            f = rf[2 * r + i]
            if f >= 0:
                Q[f, r] = rw[2 * r + i]
    return Q


def test_pole_map_matches_oracle_transform():
    pts = S.sphere_generatrix(1.0, 12)
    body = OB.Body(pts)
    for m in (-3, -1, 0, 1, 2):
        rf, rw, nred = B.pole_map(pts, m)
        Q = _q_from_map(rf, rw, nred, len(pts))
        np.testing.assert_array_equal(Q, OB.pole_transform(body, m))


def test_mode_limits_follow_reference_rule():
    cap, bw = B.mode_limits(25.0, 1.0, [0, 90], None)
    assert bw == 25 and cap == 25 + max(12, int(np.ceil(4.05 * 25 ** (1 / 3) + 2)))
    assert B.mode_limits(25.0, 1.0, [0.0, 180.0], None) == (1, 1)
    assert B.mode_limits(3.0, 1.0, [30.0], 10) == (10, 2)


def test_pair_routing_and_point_rules_match_oracle():
    """The product's near-pair routing and point sets equal the oracle's restatement of the
    reference's (graded cells for self / adjacent pairs, 12 x 12 Gauss for the others)."""
    from grim_20261007_b200.bor import rules
    G = np.load(os.path.join(GOLDEN, 'ref_bor_modes.npz'))
    for pts in (S.sphere_generatrix(1.0, 20), S.ogive_generatrix(3.0, 22.0, 30), G['graded_points']):
        np.testing.assert_array_equal(rules.pair_classes(pts), OB.Body(pts).pair_classes())
    rule, starts = rules.near_rules()
    parts = [OB.cell_points('diag'), OB.cell_points('corner10'), OB.cell_points('corner01'), OB.regular_points()]
    for i, (s, sq, w) in enumerate(parts):
        np.testing.assert_array_equal(rule[starts[i]:starts[i + 1]], np.stack([s, sq, w], axis=1))
    assert starts[-1] == len(rule)


def test_mirror_map_is_a_signed_involution_matching_the_oracle_matrices():
    """The mirror map of a symmetric body is an involution with J_t -> -J_t, J_phi -> J_phi,
    and the oracle's reduced mode matrices satisfy Z = R Z R with it; a body that is not
    symmetric has no map."""
    pts = S.ogive_generatrix(3.0, 22.0, 18)
    body = OB.Body(pts)
    asm = OB.Assembler(body, 5.0, 3, mfie=True)
    for m in (0, 1, -1, 2):
        target, sign = B.mirror_map(pts, m)
        n = len(target)
        assert np.array_equal(target[target], np.arange(n)) and np.array_equal(sign[target], sign)
        R = np.zeros((n, n))
        R[np.arange(n), target] = sign
        Q = OB.pole_transform(body, m)
        Zr = Q.conj().T @ asm.cfie_matrix(m) @ Q
        assert np.max(np.abs(R @ Zr @ R - Zr)) <= 1e-13 * np.max(np.abs(Zr))
        p1, p2, s, fe, fo = B.mirror_parts(target, sign)
        assert 2 * len(p1) + len(fe) + len(fo) == n
    bent = pts.copy()
    bent[3, 0] *= 1.01
    assert B.mirror_map(bent, 0) is None


@pytest.mark.parametrize('kwargs, exc', [
    (dict(formulation='pmchwt'), ValueError),
    (dict(formulation='cfie', cfie_alpha=1.0), ValueError),
    (dict(formulation='auto', cfie_alpha=float('nan')), ValueError),
    (dict(zs=50.0), NotImplementedError),
    (dict(sheet_zs=10.0), NotImplementedError),
    (dict(gauss_order=5), ValueError),
])
def test_solve_bor_rejects_arguments_before_any_device_work(kwargs, exc):
    """solve_bor refuses unsupported formulations, CFIE weights outside (0, 1), impedance and
    sheet models and other far-pair Gauss orders with the reference's error types, before it
    needs a device."""
    with pytest.raises(exc):
        B.solve_bor(S.sphere_generatrix(1.0, 12), 3e8, [0.0, 90.0], **kwargs)


def test_validate_generatrix_rules():
    pts = S.sphere_generatrix(1.0, 8)
    out = B.validate_generatrix(pts)
    assert out[0, 0] == 0.0 and out[-1, 0] == 0.0
    with pytest.raises(ValueError):
        B.validate_generatrix(pts[:2])
    bad = pts.copy()
    bad[3, 0] = -0.5
    with pytest.raises(ValueError):
        B.validate_generatrix(bad)
    dup = np.vstack([pts[:3], pts[2:]])
    with pytest.raises(ValueError):
        B.validate_generatrix(dup)


def test_mixed_requests_pick_the_precision_per_mode():
    """Mixed precision only for mode systems of at least MIXED_MIN_ORDER unknowns below
    MIXED_MODE_FRACTION k rho_max; FP64 requests stay FP64."""
    from types import SimpleNamespace
    from grim_20261007_b200.bor import solver as bs
    dev = SimpleNamespace(k=25.0, nodes=np.array([[0.0, 1.0], [1.0, 0.0], [0.0, -1.0]]))
    assert bs.mode_precision(dev, 3, 4000, 'double') == 'double'
    assert bs.mode_precision(dev, 3, 4000, 'mixed') == 'mixed'
    assert bs.mode_precision(dev, 18, 4000, 'mixed') == 'double'   # >= 0.7 k rho_max
    assert bs.mode_precision(dev, 3, 800, 'mixed') == 'double'     # below the order threshold


def test_release_gate_decisions():
    """The per-mode release gate's host rules (reference bor/factor.py:302-355): limits per
    precision, the pass test, and the refinement stop rule."""
    from grim_20261007_b200.bor import solver as B
    assert B.BOR_LINEAR_BACKWARD_ERROR_MAX == 1e-12 and B.BOR_LINEAR_RESIDUAL_MAX == 1e-8
    assert B.release_limit('double', 1e-10) == 1e-12
    assert B.release_limit('mixed', 1e-10) == 1e-10
    assert B.release_limit('mixed', 1e-14) == 1e-12
    assert B.gate_decision(1e-13, 1e-9, 1e-12)
    assert not B.gate_decision(2e-12, 1e-9, 1e-12)
    assert not B.gate_decision(1e-13, 2e-8, 1e-12)  # the relative residual alone sends it to refinement
    assert not B.gate_decision(float('nan'), 0.0, 1e-12)
    assert not B.gate_decision(0.0, float('inf'), 1e-12)
    assert B.refinement_continues((1e-10, 1e-6), (1e-11, 1e-6))   # backward error fell
    assert B.refinement_continues((1e-10, 1e-6), (1e-9, 1e-7))    # residual fell
    assert not B.refinement_continues((1e-10, 1e-6), (1e-10, 1e-6))
    assert not B.refinement_continues((1e-10, 1e-6), (2e-10, 2e-6))


def test_condition_gate_messages():
    """The reference's condition release test (bor/factor.py:224-229) on host values."""
    from grim_20261007_b200.bor import solver as B
    assert B.BOR_CONDITION_EST_MAX == 1e12
    B.condition_gate([0, 1], [1.0, 9e11])
    with pytest.raises(RuntimeError, match='m=3 estimated 1-norm condition .* exceeds the release limit'):
        B.condition_gate([2, 3], [5.0, 2e12])
    for bad in (float('nan'), float('inf'), 0.0):
        with pytest.raises(RuntimeError, match='m=4 condition estimation failed'):
            B.condition_gate([4], [bad])


def test_finish_modes_decisions_without_a_device(monkeypatch):
    """The per-mode path's gate bookkeeping (``_finish_modes``) on host stand-ins: the
    condition gate is applied to every mode first, then exactly the modes whose measures
    miss their release limits are solved again (``_redo_mode``), a mixed one marked as an
    LU fallback."""
    import torch

    class Lib:
        @staticmethod
        def grim_synchronize(h):
            return 0

    class Ctx:
        lib, h = Lib(), None

    redone = []

    def fake_redo(dev, m, th, tol, ctx, monitor_cond):
        redone.append(m)
        return torch.full((2,), float(m)), {'backward_error': 1e-15, 'relative_residual': 1e-14,
                                            'gate_refinement_steps': 1, 'condition_est': 10.0}

    monkeypatch.setattr(B, '_redo_mode', fake_redo)

    def res(m, berr, rel, prec, cond):
        return (torch.zeros(2), {'fp64_fallback': False},
                {'precision': prec, 'maxes': torch.tensor([berr, rel], dtype=torch.float64),
                 'cond': torch.tensor([cond], dtype=torch.float64)})

    results = [res(0, 1e-15, 1e-12, 'double', 5.0),      # released
               res(1, 2e-12, 1e-12, 'double', 5.0),      # backward error above 1e-12: redone
               res(2, 5e-11, 1e-12, 'mixed', 5.0),       # mixed at its 1e-10 target: released
               res(3, 1e-15, 3e-8, 'mixed', 5.0)]        # relative residual above 1e-8: redone
    outs = B._finish_modes(None, [0, 1, 2, 3], None, results, 1e-10, Ctx(), True)
    assert redone == [1, 3]
    assert [float(p[0]) for p, _t in outs] == [0.0, 1.0, 0.0, 3.0]
    assert 'gate_lu_fallback' in outs[3][1] and 'gate_lu_fallback' not in outs[1][1]
    assert outs[0][1]['backward_error'] == 1e-15 and outs[0][1]['condition_est'] == 5.0
    # the condition gate comes first: a mode over the limit raises before any re-solve
    redone.clear()
    bad = [res(0, 2e-12, 1e-12, 'double', 5.0), res(1, 1e-15, 1e-12, 'double', 2e12)]
    with pytest.raises(RuntimeError, match='m=1 estimated 1-norm condition'):
        B._finish_modes(None, [0, 1], None, bad, 1e-10, Ctx(), True)
    assert redone == []
