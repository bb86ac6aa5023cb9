"""The 2-D linear-Galerkin near-block oracle against the reference's own self and touching
blocks (tests/golden/galerkin_near.npz, made by tests/golden/make_galerkin_near_golden.py)."""
import os

import numpy as np
import pytest

from oracle import galerkin2d as G
from tests.conftest import GOLDEN

F = np.load(os.path.join(GOLDEN, 'galerkin_near.npz'))


@pytest.mark.parametrize('i', range(len(F['self_k'])))
def test_self_block_matches_reference(i):
    """Self single-layer blocks: the series up to |k l| = 8, the composite rule beyond."""
    got = G.self_block(F['self_length'][i], F['self_k'][i])
    ref = F['self_s'][i]
    assert np.max(np.abs(got - ref)) <= 1e-13 * np.max(np.abs(ref))


def test_self_block_series_on_a_sub_interval_is_the_parent_basis_projection():
    """A sub-interval's series block in the parent basis equals the full block's series for
    a sub-interval [0, 1] of a shorter element, mapped by the hat functions."""
    length, k = 0.2, 15.0
    sub = G.self_block_series(length, k, 0.25, 0.75)
    local = G.self_block_series(0.5 * length, k)
    t = np.array([[0.75, 0.25], [0.25, 0.75]])
    assert np.allclose(sub, t @ local @ t.T, rtol=1e-14, atol=1e-16)


@pytest.mark.parametrize('i', range(len(F['touch_k'])))
def test_touching_blocks_match_reference(i):
    ends = F['touch_ends'][i]
    po, ps = ends[:2], ends[2:]

    def normal(p):
        t = (p[1] - p[0]) / np.hypot(*(p[1] - p[0]))
        return np.array([t[1], -t[0]])

    s_blk, k_blk = G.touching_blocks(po, ps, normal(po), normal(ps), bool(F['touch_obs_start'][i]),
                                     bool(F['touch_src_start'][i]), float(F['touch_k'][i]),
                                     bool(F['touch_obs_deriv'][i]))
    s_ref, k_ref = F['touch_s'][i], F['touch_kd'][i]
    assert np.max(np.abs(s_blk - s_ref)) <= 1e-13 * np.max(np.abs(s_ref))
    # K' of collinear elements is zero up to rounding: scale the bound by |S| k as well
    scale = max(np.max(np.abs(k_ref)), np.max(np.abs(s_ref)) * float(F['touch_k'][i]))
    assert np.max(np.abs(k_blk - k_ref)) <= 1e-13 * scale


def _ring():
    pts = F['ring_points']
    n = len(pts)
    ends = [(pts[i], pts[(i + 1) % n]) for i in range(n)]

    def normal(e):
        t = (e[1] - e[0]) / np.hypot(*(e[1] - e[0]))
        return np.array([t[1], -t[0]])
    return ends, [normal(e) for e in ends]


def test_adaptive_routing_matches_reference():
    """The separated-pair predicate (centre, gap and projection clauses) routes every near pair
    of the ring as the reference does."""
    ends, _normals = _ring()
    got = np.array([G.needs_adaptive(ends[i], ends[j]) for i, j in F['ring_pairs']])
    np.testing.assert_array_equal(got, F['ring_adaptive'])
    assert got.sum() > 50 and (~got).sum() > 1000


def test_box_blocks_match_reference():
    """16-point tensor S and K' blocks (source and observation normal) of the ring's box pairs."""
    ends, normals = _ring()
    box = F['ring_pairs'][~F['ring_adaptive']]
    k = float(F['ring_k'])
    for idx, (i, j) in enumerate(box):
        s_blk, kd_src = G.box_blocks(ends[i], ends[j], normals[i], normals[j], k, False)
        _s, kd_obs = G.box_blocks(ends[i], ends[j], normals[i], normals[j], k, True)
        for got, ref in ((s_blk, F['box_s'][idx]), (kd_src, F['box_kd_src'][idx]), (kd_obs, F['box_kd_obs'][idx])):
            assert np.max(np.abs(got - ref)) <= 1e-13 * max(np.max(np.abs(ref)), np.max(np.abs(F['box_s'][idx])) * k)


def test_adaptive_blocks_match_reference():
    """Close separated pairs of the ring (the reference's adaptive routing) by the bisection
    rule to 1e-9: S and K' (source and observation normal) equal the reference's."""
    ends, normals = _ring()
    close = F['ring_pairs'][F['ring_adaptive']]
    k = float(F['ring_k'])
    for idx, (i, j) in enumerate(close):
        s_blk, kd_src = G.adaptive_blocks(ends[i], ends[j], normals[i], normals[j], k, False)
        _s, kd_obs = G.adaptive_blocks(ends[i], ends[j], normals[i], normals[j], k, True)
        scale = np.max(np.abs(F['adaptive_s'][idx])) * k
        for got, ref in ((s_blk, F['adaptive_s'][idx]), (kd_src, F['adaptive_kd_src'][idx]),
                         (kd_obs, F['adaptive_kd_obs'][idx])):
            assert np.max(np.abs(got - ref)) <= 1e-13 * max(np.max(np.abs(ref)), scale)


def test_maue_blocks_match_reference():
    ends, normals = _ring()
    box = F['ring_pairs'][~F['ring_adaptive']]
    k = float(F['ring_k'])
    for idx, (i, j) in enumerate(box):
        lo, ls = (float(np.hypot(*(e[1] - e[0]))) for e in (ends[i], ends[j]))
        got = G.maue_block(F['box_s'][idx], k, normals[i], normals[j], lo, ls)
        ref = F['box_maue'][idx]
        assert np.max(np.abs(got - ref)) <= 1e-14 * np.max(np.abs(ref))


@pytest.mark.parametrize('tag,k', [('k30', 30.0), ('k4', 4.0)])
def test_whole_ring_operators_match_reference(tag, k):
    """The ring's node-based S and K' from element blocks (far pairs at the tile's graded
    order, near pairs by their routes) equal the reference's own assembly."""
    ends, normals = _ring()
    n = len(ends)
    node_ids = [(i, (i + 1) % n) for i in range(n)]
    S, Kp = G.assemble_single_tile(ends, node_ids, normals, k, n)
    for got, ref in ((S, F[f'ring_S_{tag}']), (Kp, F[f'ring_K_{tag}'])):
        assert np.max(np.abs(got - ref)) <= 1e-14 * np.max(np.abs(ref))
