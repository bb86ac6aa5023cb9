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


AIRFOIL = np.load(os.path.join(GOLDEN, 'ref_airfoil.npz'))


def _amplitudes(res, export=None):
    rows = [r for r in res['samples'] if export is None or r.get('polarization') == export]
    return (np.array([complex(r['rcs_amp_real'], r['rcs_amp_imag']) for r in rows]),
            np.array([r['rcs_linear'] for r in rows]))


def test_c1_cylinder_through_the_public_entry(ctx):
    """Config 1 through solve_monostatic_rcs_2d_single_polarization: the reference's own
    amplitudes (1e-10), the Mie series (1e-3 dB) and the FP64 gate."""
    from oracle import mie
    from grim_20261007_b200.twod.solver import solve_monostatic_rcs_2d_single_polarization
    g = np.load(os.path.join(GOLDEN, 'ref_cylinder_c1.npz'))
    snap = S.snapshot_from_polygons([S.circle(1.0, 200)])
    for pol in ('TM', 'TE'):
        res = solve_monostatic_rcs_2d_single_polarization(snap, [float(g['frequency_ghz'])], list(g['angles']), pol,
                                                          geometry_units='meters', strict_quality_gate=True)
        amp, sig = _amplitudes(res)
        assert np.max(np.abs(amp - g[f'amp_{pol}']) / np.abs(g[f'amp_{pol}'])) <= 1e-10
        assert abs(10 * np.log10(sig[0] / mie.cylinder_sigma(1.0, float(g['k']), pol))) <= 1e-3
        assert max(r['linear_residual'] for r in res['samples']) <= 1e-12
        assert 'Galerkin' in res['metadata']['formulation']


@pytest.mark.parametrize('n', [int(x) for x in AIRFOIL['sizes']])
def test_airfoil_matches_the_reference_solver(ctx, n):
    """The headline geometry (seeded NACA 00tt, blunt trailing edge, cosine spacing, lambda/10,
    720 angles) through solve_monostatic_rcs_2d: both channels' complex amplitudes equal the
    reference solver's (tests/golden/ref_airfoil.npz) to 1e-9 of the peak amplitude in FP64;
    the mixed-precision path is within 0.05 dB of the reference wherever sigma is within
    40 dB of its peak."""
    from grim_20261007_b200.execution import linear_precision
    from grim_20261007_b200.twod.solver import solve_monostatic_rcs_2d
    v, k, f, _t = S.airfoil_case(0, n)
    assert abs(k - float(AIRFOIL[f'n{n}_k'])) <= 1e-12 * k
    snap = S.snapshot_from_polygons([v])
    ang = list(AIRFOIL['angles'])
    r64 = solve_monostatic_rcs_2d(snap, [f / 1e9], ang, geometry_units='meters')
    with linear_precision('mixed'):
        r32 = solve_monostatic_rcs_2d(snap, [f / 1e9], ang, geometry_units='meters')
    for pol, export in (('TE', 'VV'), ('TM', 'HH')):
        ref_amp, ref_sig = AIRFOIL[f'n{n}_amp_{pol}'], AIRFOIL[f'n{n}_sigma_{pol}']
        a64, s64 = _amplitudes(r64, export)
        _a32, s32 = _amplitudes(r32, export)
        assert np.max(np.abs(a64 - ref_amp)) <= 1e-9 * np.max(np.abs(ref_amp)), pol
        db = 10 * np.log10(ref_sig)
        mask = db > db.max() - 40
        assert np.max(np.abs(10 * np.log10(s64[mask] / ref_sig[mask]))) <= 1e-6, pol
        assert np.max(np.abs(10 * np.log10(s32[mask] / ref_sig[mask]))) <= 0.05, pol


@pytest.mark.parametrize('pol', ['TM', 'TE'])
def test_gated_solve_pivots_like_lapack_and_falls_back(ctx, pol):
    """The airfoil's combined-field matrix factors with partial pivoting into LAPACK's pivots
    and meets the reference's 1e-12 backward-error gate without refinement; a static-pivot
    solve of a system whose leading entry is zero falls back to the certified factorization."""
    import ctypes
    import scipy.linalg as sla
    from grim_20261007_b200 import _lib
    from grim_20261007_b200.device import context, ptr, to_device_colmajor, to_host_matrix
    from grim_20261007_b200.twod import operators as ops
    from grim_20261007_b200.twod.galerkin import GalerkinBody
    v, k, _f, _t = S.airfoil_case(2, 512)
    body = GalerkinBody([v])
    z = body.fill_matrix(k, pol)
    ang = torch.as_tensor(np.arange(0.0, 360.0, 3.0), device='cuda')
    x = body.rhs_matrix(k, pol, ang)
    b = x.clone()
    st, berr = ops.solve_guarded(z, x, pivot='partial')
    assert float(berr.max()) <= 1e-12 and st['refinement_steps'] == 0 and not st['gate_fallback']
    assert float(ops.backward_error(z, x, b).max()) <= 1e-12
    c = context()
    lu = z.clone()
    ipiv = torch.zeros(body.n, dtype=torch.int32, device='cuda')
    info = ctypes.c_int(-1)
    _lib.check(c.lib.grim_set_tuning(c.h, _lib.TUNE_PIVOT, _lib.PIVOT_PARTIAL))
    try:
        _lib.check(c.lib.grim_zgetrf(c.h, body.n, ptr(lu), body.n, ptr(ipiv), ctypes.byref(info)))
    finally:
        c.lib.grim_set_tuning(c.h, _lib.TUNE_PIVOT, _lib.PIVOT_CERTIFIED)
    lu_ref, piv_ref = sla.lu_factor(to_host_matrix(z))
    np.testing.assert_array_equal(ipiv.cpu().numpy(), piv_ref + 1)
    assert np.max(np.abs(to_host_matrix(lu) - lu_ref)) <= 1e-11 * np.max(np.abs(lu_ref))
    rng = np.random.default_rng(1)
    a = rng.standard_normal((96, 96)) + 1j * rng.standard_normal((96, 96))
    a[0, 0] = 0.0
    rhs = rng.standard_normal((96, 3)) + 0j
    x2 = to_device_colmajor(rhs)
    st2, berr2 = ops.solve_guarded(to_device_colmajor(a), x2, pivot='static')
    assert st2['gate_fallback'] and float(berr2.max()) <= 1e-12
    np.testing.assert_allclose(x2.cpu().numpy().T, np.linalg.solve(a, rhs), rtol=1e-10, atol=1e-12)


def test_condition_number_and_quality_gate_through_the_public_entry(ctx):
    """compute_condition_number=True reports the equilibrated condition estimate of every
    system (condition_est_max / mean, the estimator's name) and the reference's quality gate
    checks it: a limit below it fails the strict gate with the reference's message."""
    import pytest as _pt
    from grim_20261007_b200 import synthetic as S
    from grim_20261007_b200.twod.solver import solve_monostatic_rcs_2d_single_polarization as solve1
    v = S.naca_symmetric(0.12, 120)
    snap = S.snapshot_from_polygons([v])
    ang = list(np.arange(0.0, 180.0, 10.0))
    out = solve1(snap, [0.9, 1.4], ang, 'TE', geometry_units='meters', compute_condition_number=True)
    meta = out['metadata']
    assert meta['condition_est_computed'] and meta['condition_estimator'] == 'equilibrated_1norm_lu_hager_higham'
    assert 1.0 <= meta['condition_est_max'] < 1e6 and meta['condition_est_mean'] <= meta['condition_est_max']
    gate = meta['quality_gate']
    assert gate['passed'] and gate['certification_scope'] == 'discrete_linear_system_residual_and_condition'
    with _pt.raises(ValueError, match='condition_est_max'):
        solve1(snap, [0.9], ang, 'TE', geometry_units='meters', compute_condition_number=True,
               quality_thresholds={'condition_est_max': 1.0})
    plain = solve1(snap, [0.9], ang, 'TE', geometry_units='meters')
    assert not plain['metadata']['condition_est_computed']
    assert plain['metadata']['quality_gate']['certification_scope'] == 'discrete_linear_system_residual_only'


@pytest.mark.parametrize('pol', ['TM', 'TE'])
def test_tournament_pivoting_meets_the_gate_on_the_airfoil(ctx, pol):
    """Tournament pivoting (tslu.cuh) of the linear-Galerkin systems: on the
    2048-element airfoil the FP64 solve meets the reference's 1e-12 backward-error gate and
    equals the partial-pivoting (LAPACK-pivot) solution to 1e-10; the mixed solve through a
    complex64 tournament factorization refines to the same solution."""
    from grim_20261007_b200.twod import operators as ops
    from grim_20261007_b200.twod.galerkin import GalerkinBody
    v, k, _f, _t = S.airfoil_case(0, 2048)
    body = GalerkinBody([v])
    z = body.fill_matrix(k, pol)
    ang = torch.as_tensor(np.arange(0.0, 360.0, 2.0), device='cuda')
    b = body.rhs_matrix(k, pol, ang)
    xt, xp, xm = b.clone(), b.clone(), b.clone()
    st, berr = ops.solve_guarded(z, xt, pivot='tournament')
    assert float(berr.max()) <= 1e-12 and not st['gate_fallback'], st
    _st, _b = ops.solve_guarded(z, xp, pivot='partial')
    scale = float(xp.abs().max())
    assert float((xt - xp).abs().max()) <= 1e-10 * scale
    ops.solve_inplace(z, xm, 'mixed', tol=1e-12, stop='berr', pivot='tournament', tuned=False)
    assert float((xm - xp).abs().max()) <= 1e-9 * scale


def test_public_results_export_to_grim(ctx, tmp_path):
    """A co-polarised and a single-polarisation solve of the C1 cylinder export to `.grim`
    (the reference's archive format) and read back with their own amplitudes."""
    from grim_20261007_b200 import grimfile
    from grim_20261007_b200.twod.solver import (solve_monostatic_rcs_2d,
                                                solve_monostatic_rcs_2d_single_polarization as solve1)
    snap = S.snapshot_from_polygons([S.circle(1.0, 200)])
    ang = list(np.arange(0.0, 360.0, 10.0))
    both = solve_monostatic_rcs_2d(snap, [0.4, 0.5], ang, geometry_units='meters')
    path = grimfile.export_result_to_grim(both, str(tmp_path / 'co'))[0]
    back = grimfile.load_grim_npz(path)
    assert list(back['polarizations']) == ['VV', 'HH'] and back['rcs_amp_real'].shape == (36, 1, 2, 2)
    for p, pol in enumerate(('VV', 'HH')):
        rows = [r for r in both['samples'] if r['polarization'] == pol]
        for r in rows:
            i = ang.index(r['theta_scat_deg'])
            j = [0.4, 0.5].index(r['frequency_ghz'])
            assert back['rcs_amp_real'][i, 0, j, p] == r['rcs_amp_real']
            assert back['rcs_amp_imag'][i, 0, j, p] == r['rcs_amp_imag']
    one = solve1(snap, [0.4], ang, 'TM', geometry_units='meters')
    back1 = grimfile.load_grim_npz(grimfile.export_result_to_grim(one, str(tmp_path / 'tm.grim'), format_version=1)[0])
    assert list(back1['polarizations']) == ['HH'] and back1['rcs_power'].dtype == np.float32
