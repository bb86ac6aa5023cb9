"""The 2-D Galerkin oracle's whole combined PEC system against the reference's own dense
systems as they reach its dense-solver hook (tests/golden/ref_dense_system.npz, made by
tests/golden/make_golden.py): the operators S, K', W and the mass from element blocks, the
combined routes S + gamma (D + M/2) (TM) and K' - M/2 - gamma W (TE), and the plane-wave
right-hand sides, on the reference's drawn circles."""
import os

import numpy as np
import pytest

from oracle import galerkin2d as G
from tests.conftest import GOLDEN

F = np.load(os.path.join(GOLDEN, 'ref_dense_system.npz'))
ANGLES = [0.0, 30.0, 90.0, 135.0, 200.0, 300.0]   # the captured solves' incidence angles
CASES = {'cyl64_ka1': (0.1, 64, 1.0), 'cyl64_ka2p4': (0.1, 64, 2.404825557695773), 'cyl96_ka5': (0.1, 96, 5.0)}
_ASSEMBLED = {}


def _system(name, pol):
    radius, count, ka = CASES[name]
    theta = np.linspace(0.0, -2.0 * np.pi, count + 1)[:-1]          # drawn clockwise, as captured
    nodes = G.drawn_to_solver_contour(np.stack([radius * np.cos(theta), radius * np.sin(theta)], axis=1))
    k = ka / radius
    if name not in _ASSEMBLED:
        n = len(nodes)
        ends = [(nodes[i], nodes[(i + 1) % n]) for i in range(n)]
        normals = [np.array([-(b - a)[1], (b - a)[0]]) / np.hypot(*(b - a)) for a, b in ends]
        _ASSEMBLED[name] = G.assemble_single_tile(ends, [(i, (i + 1) % n) for i in range(n)], normals, k, n,
                                                  hypersingular=True)
    return G.pec_combined_system(nodes, k, ANGLES, pol, operators=_ASSEMBLED[name])


@pytest.mark.parametrize('pol', ['TM', 'TE'])
@pytest.mark.parametrize('name', list(CASES))
def test_combined_system_matches_reference_hook(name, pol):
    A, b = _system(name, pol)
    ref_a, ref_b = F[f'{name}_{pol}_a'], F[f'{name}_{pol}_b']
    assert A.shape == ref_a.shape and b.shape == ref_b.shape
    assert np.max(np.abs(A - ref_a)) <= 1e-13 * np.max(np.abs(ref_a))
    assert np.max(np.abs(b - ref_b)) <= 1e-13 * np.max(np.abs(ref_b))
    # and the solution the reference's LAPACK path returned for it
    x = np.linalg.solve(A, b)
    ref_x = F[f'{name}_{pol}_x']
    assert np.max(np.abs(x - ref_x)) <= 1e-9 * np.max(np.abs(ref_x))


def test_combined_system_rejects_unknown_polarization():
    nodes = G.drawn_to_solver_contour(np.array([[1.0, 0.0], [0.0, -1.0], [-1.0, 0.0], [0.0, 1.0]]))
    ops = tuple(np.eye(4, dtype=complex) for _ in range(3))
    with pytest.raises(ValueError):
        G.pec_combined_system(nodes, 1.0, [0.0], 'TX', operators=ops)


def test_drawn_contour_is_reversed_about_its_first_point():
    drawn = np.arange(10.0).reshape(5, 2)
    np.testing.assert_array_equal(G.drawn_to_solver_contour(drawn), drawn[[0, 4, 3, 2, 1]])


def test_combined_rows_remove_the_interior_resonance():
    """At ka = 2.405 (the first zero of J0, a TM interior resonance of the circle) the bare
    single layer degrades against the same mesh at ka = 1 (about 3x in condition number),
    the combined S + gamma (D + M/2) stays where it was (within 5%) and about 80x better."""
    cond = {}
    for name in ('cyl64_ka1', 'cyl64_ka2p4'):
        A, _b = _system(name, 'TM')
        cond[name] = np.linalg.cond(_ASSEMBLED[name][0]), np.linalg.cond(A)
    (s_off, a_off), (s_res, a_res) = cond['cyl64_ka1'], cond['cyl64_ka2p4']
    assert s_res > 2.5 * s_off
    assert a_res < 1.2 * a_off
    assert s_res > 50.0 * a_res


MIE = np.load(os.path.join(GOLDEN, 'mie_cylinder.npz'))


@pytest.mark.parametrize('pol', ['TM', 'TE'])
@pytest.mark.parametrize('name', list(CASES))
def test_combined_solution_scatters_like_the_mie_series(name, pol):
    """Fill, solve and far field of the oracle's own combined system: the monostatic width of
    the polygonal circle is the reference's Mie series (sigma / a depends on ka only) to the
    discretisation error, 0.2% here, at every incidence angle."""
    radius, count, ka = CASES[name]
    A, b = _system(name, pol)
    theta = np.linspace(0.0, -2.0 * np.pi, count + 1)[:-1]
    nodes = G.drawn_to_solver_contour(np.stack([radius * np.cos(theta), radius * np.sin(theta)], axis=1))
    sigma = G.pec_combined_sigma(nodes, ka / radius, ANGLES, np.linalg.solve(A, b))
    i = int(np.argmin(np.abs(MIE['ka'] - ka)))
    assert abs(MIE['ka'][i] - ka) < 1e-9
    mie = radius * MIE['sigma'][['TM', 'TE'].index(pol), i]
    np.testing.assert_allclose(sigma, mie, rtol=2e-3)
