"""GPU linear-Galerkin combined-field fill, loads and far field against the oracle and the
reference's own dense systems and solutions.

The GPU picks its far Gauss order per 32 x 32 element tile from the reference's calibrated
table, the reference per assembly tile; the table holds every far block within 1e-12 of a
converged rule, so matrices agree to 1e-12 of their largest entry (1e-13 where the
reference assembled the contour as one tile with the same worst pair)."""
import os

import numpy as np
import pytest

from oracle import galerkin2d as G
from grim_20261007_b200 import synthetic as S
from tests.conftest import GOLDEN

pytestmark = pytest.mark.gpu
torch = pytest.importorskip('torch')

DENSE = np.load(os.path.join(GOLDEN, 'ref_dense_system.npz'))
DENSE_ANGLES = [0.0, 30.0, 90.0, 135.0, 200.0, 300.0]
DENSE_CASES = {'cyl64_ka1': (0.1, 64, 1.0), 'cyl64_ka2p4': (0.1, 64, 2.404825557695773), 'cyl96_ka5': (0.1, 96, 5.0)}


@pytest.fixture(scope='module')
def ctx():
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from grim_20261007_b200.device import context
    return context()


def _drawn_circle(radius, count):
    theta = np.linspace(0.0, -2.0 * np.pi, count + 1)[:-1]
    return np.stack([radius * np.cos(theta), radius * np.sin(theta)], axis=1)


def _jittered_ring(seed, count):
    rng = np.random.default_rng(seed)
    theta = -2.0 * np.pi * (np.arange(count) + 0.3 * rng.uniform(-1, 1, count)) / count
    r = 1.0 + 0.05 * rng.uniform(-1, 1, count)
    return np.stack([r * np.cos(theta), r * np.sin(theta)], axis=1)


def _oracle_operators(drawn, k):
    nodes = G.drawn_to_solver_contour(drawn)
    n = len(nodes)
    ends = [(nodes[i], nodes[(i + 1) % n]) for i in range(n)]
    normals = [np.array([-(b - a)[1], (b - a)[0]]) / np.hypot(*(b - a)) for a, b in ends]
    return nodes, G.assemble_single_tile(ends, [(i, (i + 1) % n) for i in range(n)], normals, k, n, hypersingular=True)


def _gpu_matrix(body, k, pol, complex64=False):
    from grim_20261007_b200.device import to_host_matrix
    z = to_host_matrix(body.fill_matrix(k, pol, complex64=complex64))
    body.check_status()
    return z


# Contours with near pairs of every route: a jittered ring (touching and fixed-rule pairs),
# a 64-element cosine-spaced airfoil with a blunt trailing edge (adaptive close pairs at the
# leading and trailing edges), a coarse circle whose elements are longer than the self
# series' range (composite self blocks).
CONTOURS = {
    'ring60': lambda: (_jittered_ring(3, 60), 6.0),
    'naca64': lambda: (S.naca_symmetric(0.12, 64), 2 * np.pi / (S.polygon_perimeter(S.naca_symmetric(0.12, 64)) * 10 / 64)),
    'coarse_circle10': lambda: (_drawn_circle(1.0, 10), 14.0),
}


@pytest.mark.parametrize('name', list(CONTOURS))
def test_near_pair_structure_matches_the_reference_routing(ctx, name):
    from grim_20261007_b200.twod.galerkin import GalerkinBody
    drawn, _k = CONTOURS[name]()
    body = GalerkinBody([drawn])
    nodes = G.drawn_to_solver_contour(drawn)
    n = len(nodes)
    ends = [(nodes[i], nodes[(i + 1) % n]) for i in range(n)]
    lengths = np.array([np.hypot(*(b - a)) for a, b in ends])
    centres = np.array([0.5 * (a + b) for a, b in ends])
    row_off = body.row_off.cpu().numpy()
    col = body.col.cpu().numpy()[:body.nnz]
    route = body.route.cpu().numpy()[:body.nnz]
    for e in range(n):
        want_cols, want_routes = [], []
        for f in range(n):
            share = bool({e, (e + 1) % n} & {f, (f + 1) % n})
            ratio = np.hypot(*(centres[e] - centres[f])) / max(lengths[e], lengths[f])
            if e != f and not share and ratio >= 3.0:
                continue
            want_cols.append(f)
            want_routes.append(0 if e == f else 1 if share else 3 if G.needs_adaptive(ends[e], ends[f]) else 2)
        got = slice(row_off[e], row_off[e + 1])
        assert col[got].tolist() == want_cols
        assert route[got].tolist() == want_routes
    if name == 'naca64':
        assert np.any(route == 3), 'the airfoil must exercise the adaptive rule'


@pytest.mark.parametrize('pol', ['TM', 'TE'])
@pytest.mark.parametrize('name', list(CONTOURS))
def test_fill_matches_oracle_operators(ctx, name, pol):
    from grim_20261007_b200.twod.galerkin import GalerkinBody
    drawn, k = CONTOURS[name]()
    nodes, ops_ = _oracle_operators(drawn, k)
    A, _b = G.pec_combined_system(nodes, k, [0.0], pol, operators=ops_)
    z = _gpu_matrix(GalerkinBody([drawn]), k, pol)
    assert np.max(np.abs(z - A)) <= 1e-12 * np.max(np.abs(A))


@pytest.mark.parametrize('pol', ['TM', 'TE'])
@pytest.mark.parametrize('name', list(DENSE_CASES))
def test_fill_and_loads_match_the_reference_dense_systems(ctx, name, pol):
    """The matrix and right-hand sides the reference hands to its dense solver (captured at
    its GPU hook) on its drawn circles, including the first interior resonance."""
    from grim_20261007_b200.twod.galerkin import GalerkinBody
    from grim_20261007_b200.device import to_host_matrix
    radius, count, ka = DENSE_CASES[name]
    k = ka / radius
    body = GalerkinBody([_drawn_circle(radius, count)])
    ref_a, ref_b = DENSE[f'{name}_{pol}_a'], DENSE[f'{name}_{pol}_b']
    z = _gpu_matrix(body, k, pol)
    assert np.max(np.abs(z - ref_a)) <= 1e-13 * np.max(np.abs(ref_a))
    ang = torch.as_tensor(np.array(DENSE_ANGLES), device='cuda')
    b = body.rhs_matrix(k, pol, ang).cpu().numpy().T
    assert np.max(np.abs(b - ref_b)) <= 1e-13 * np.max(np.abs(ref_b))
    bt = to_host_matrix(body.rhs_matrix(k, pol, ang))
    np.testing.assert_array_equal(bt, b)


def test_far_field_matches_oracle(ctx):
    from grim_20261007_b200.twod.galerkin import GalerkinBody
    drawn, k = CONTOURS['naca64']()
    body = GalerkinBody([drawn])
    rng = np.random.default_rng(5)
    ang = np.arange(0.0, 360.0, 7.5)
    x = rng.standard_normal((body.n, len(ang))) + 1j * rng.standard_normal((body.n, len(ang)))
    xt = torch.as_tensor(np.ascontiguousarray(x.T), device='cuda')
    amp = body.far_amplitude(k, torch.as_tensor(ang, device='cuda'), xt).cpu().numpy()
    ref = G.pec_combined_amplitude(G.drawn_to_solver_contour(drawn), k, ang, x)
    assert np.max(np.abs(amp - ref)) <= 1e-13 * np.max(np.abs(ref))
    amp32 = body.far_amplitude(k, torch.as_tensor(ang, device='cuda'), xt.to(torch.complex64)).cpu().numpy()
    assert np.max(np.abs(amp32 - ref)) <= 1e-6 * np.max(np.abs(ref))


@pytest.mark.parametrize('pol', ['TM', 'TE'])
def test_c1_cylinder_amplitudes_match_the_reference_solver(ctx, pol):
    """End to end on the reference's 200-element a = 1 m cylinder at ka = 10, 360 angles:
    the reference's stored complex amplitudes (its solver, tests/golden/ref_cylinder_c1.npz)."""
    from grim_20261007_b200.twod import operators as ops
    from grim_20261007_b200.twod.galerkin import GalerkinBody
    g = np.load(os.path.join(GOLDEN, 'ref_cylinder_c1.npz'))
    body = GalerkinBody([S.circle(1.0, 200)])
    res = ops.monostatic_solve(body, float(g['k']), g['angles'], pol, precision='double')
    amp = res['amplitude'].cpu().numpy()
    ref = g[f'amp_{pol}']
    assert np.max(np.abs(amp - ref) / np.abs(ref)) <= 1e-10
    assert float(res['telemetry']['backward_error_dev'].max()) <= 1e-12


@pytest.mark.parametrize('pol', ['TM', 'TE'])
def test_complex64_fill_is_the_rounded_fp64_fill(ctx, pol):
    from grim_20261007_b200.twod.galerkin import GalerkinBody
    drawn, k = CONTOURS['naca64']()
    body = GalerkinBody([drawn])
    z64 = _gpu_matrix(body, k, pol)
    z32 = _gpu_matrix(body, k, pol, complex64=True).astype(np.complex128)
    assert np.max(np.abs(z32 - z64)) <= 2e-6 * np.max(np.abs(z64))


def test_two_contours_are_one_system(ctx):
    """Two separate bodies: nodes of each contour numbered in turn, cross pairs far or near
    by the same rule; the matrix equals the oracle's assembly of the union of elements."""
    from grim_20261007_b200.twod.galerkin import GalerkinBody
    a = _drawn_circle(0.5, 24)
    b = _drawn_circle(0.3, 18) + np.array([1.2, 0.1])
    k = 5.0
    body = GalerkinBody([a, b])
    na, nb = G.drawn_to_solver_contour(a), G.drawn_to_solver_contour(b)
    nodes = np.concatenate([na, nb])
    ends, ids = [], []
    for base, pts in ((0, na), (len(na), nb)):
        m = len(pts)
        for i in range(m):
            ends.append((pts[i], pts[(i + 1) % m]))
            ids.append((base + i, base + (i + 1) % m))
    normals = [np.array([-(q - p)[1], (q - p)[0]]) / np.hypot(*(q - p)) for p, q in ends]
    S_, K_, W_ = G.assemble_single_tile(ends, ids, normals, k, len(nodes), hypersingular=True)
    M = G.mass_matrix(ends, ids, len(nodes))
    gamma = 1.0 / (1j * k)
    for pol, A in (('TM', S_ + gamma * (K_.T + 0.5 * M)), ('TE', K_ - 0.5 * M - gamma * W_)):
        z = _gpu_matrix(body, k, pol)
        assert np.max(np.abs(z - A)) <= 1e-12 * np.max(np.abs(A))
