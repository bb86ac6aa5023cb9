"""GPU 2-D pulse-basis fill / excitation / far field / end-to-end solve against the FP64 pulse
oracle, and the public entry points' concurrency, sweep and certification behaviour (the
default linear-Galerkin formulation; its parity tests are in test_gpu_galerkin.py)."""
import os

import numpy as np
import pytest

from oracle import mie, pulse2d as P
from grim_20261007_b200 import synthetic as S
from tests.conftest import GOLDEN

pytestmark = pytest.mark.gpu
torch = pytest.importorskip('torch')


@pytest.fixture(scope='module')
def ctx():
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from grim_20261007_b200.device import context
    return context()


def _body(v, pol):
    from grim_20261007_b200.twod import geometry as geo, operators as ops
    g = geo.panel_geometry([v])
    return ops.DeviceBody(g, geo.te_curvature_correction([v]) if pol == 'TE' else None), g


CASES = [
    ('circle200', lambda: (S.circle(1.0, 200), 10.0)),
    ('naca256', lambda: (S.naca_symmetric(0.12, 256), 2 * np.pi / (S.polygon_perimeter(S.naca_symmetric(0.12, 256)) * 10 / 256))),
    ('superellipse150', lambda: (S.superellipse(0.7, 0.3, 3.5, 150), 25.0)),
]


@pytest.mark.parametrize('case', CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize('pol', ['TM', 'TE'])
def test_fill_fp64_matches_oracle(ctx, case, pol):
    from grim_20261007_b200.twod import operators as ops
    from grim_20261007_b200.device import to_host_matrix
    v, k = case[1]()
    body, g = _body(v, pol)
    z = to_host_matrix(ops.fill(body, k, pol))
    c, t, h, n = P.panel_arrays([v])
    zr = P.fill(k, c, t, h, n, pol, te_diag=P.te_curvature_correction([v]) if pol == 'TE' else None)
    scale = np.max(np.abs(zr), axis=0)
    assert np.max(np.abs(z - zr) / scale[None, :]) <= 1e-12


@pytest.mark.parametrize('case', CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize('pol', ['TM', 'TE'])
def test_fill_complex64_matches_oracle(ctx, case, pol):
    from grim_20261007_b200.twod import operators as ops
    from grim_20261007_b200.device import to_host_matrix
    v, k = case[1]()
    body, g = _body(v, pol)
    z = to_host_matrix(ops.fill(body, k, pol, complex64=True)).astype(np.complex128)
    c, t, h, n = P.panel_arrays([v])
    zr = P.fill(k, c, t, h, n, pol, te_diag=P.te_curvature_correction([v]) if pol == 'TE' else None)
    scale = np.max(np.abs(zr), axis=0)
    # FP32 entries: a few units of FP32 rounding relative to the column scale
    assert np.max(np.abs(z - zr) / scale[None, :]) <= 2e-6


@pytest.mark.parametrize('pol', ['TM', 'TE'])
def test_rhs_and_farfield_match_oracle(ctx, pol):
    from grim_20261007_b200.twod import operators as ops
    from grim_20261007_b200.device import to_host_matrix, to_device_colmajor
    v = S.naca_symmetric(0.1, 300)
    k = 120.0
    body, g = _body(v, pol)
    ang = np.arange(0.0, 360.0, 7.5)
    ad = torch.as_tensor(ang, device='cuda')
    b = to_host_matrix(ops.rhs(body, k, pol, ad))
    c, t, h, n = P.panel_arrays([v])
    br = P.rhs(k, c, n, ang, pol)
    assert np.max(np.abs(b - br)) <= 1e-11 * np.max(np.abs(br))
    rng = np.random.default_rng(0)
    x = rng.standard_normal(br.shape) + 1j * rng.standard_normal(br.shape)
    amp = ops.farfield(body, k, ad, to_device_colmajor(x)).cpu().numpy()
    ampr = P.monostatic_amplitude(P.farfield_weights(k, c, t, h, ang), x)
    assert np.max(np.abs(amp - ampr)) <= 1e-12 * np.max(np.abs(ampr))


def test_end_to_end_c1_cylinder_fp64(ctx, monkeypatch):
    """Config 1 in the pulse formulation: PEC cylinder a=1 m, ka=10, 200 panels, 360 angles,
    TM, FP64, against the pulse oracle (and the reference / Mie to discretisation error)."""
    monkeypatch.setenv('GRIM_2D_FORMULATION', 'pulse')
    from grim_20261007_b200.twod.solver import solve_monostatic_rcs_2d_single_polarization
    g = np.load(os.path.join(GOLDEN, 'ref_cylinder_c1.npz'))
    snap = S.snapshot_from_polygons([S.circle(1.0, 200)])
    res = solve_monostatic_rcs_2d_single_polarization(snap, [float(g['frequency_ghz'])], list(g['angles']), 'TM',
                                                      geometry_units='meters', strict_quality_gate=True)
    amp = np.array([complex(s['rcs_amp_real'], s['rcs_amp_imag']) for s in res['samples']])
    sig = np.array([s['rcs_linear'] for s in res['samples']])
    o = P.solve(float(g['k']), [S.circle(1.0, 200)], g['angles'], 'TM')
    assert np.max(np.abs(amp - o['amplitude']) / np.abs(o['amplitude'])) <= 1e-10
    assert np.max(np.abs(10 * np.log10(sig / g['sigma_TM']))) <= 1e-3          # reference solver
    assert abs(10 * np.log10(sig[0] / mie.cylinder_sigma(1.0, float(g['k']), 'TM'))) <= 1e-3  # Mie
    assert max(s['linear_residual'] for s in res['samples']) <= 1e-12
    assert res['metadata']['device']


def test_end_to_end_co_polarized_and_mixed(ctx, monkeypatch):
    monkeypatch.setenv('GRIM_2D_FORMULATION', 'pulse')
    from grim_20261007_b200.execution import linear_precision
    from grim_20261007_b200.twod.solver import solve_monostatic_rcs_2d
    v, k, f, _ = S.airfoil_case(1, 512)
    snap = S.snapshot_from_polygons([v])
    ang = list(np.arange(0.0, 360.0, 2.0))
    r64 = solve_monostatic_rcs_2d(snap, [f / 1e9], ang, geometry_units='meters')
    with linear_precision('mixed'):
        r32 = solve_monostatic_rcs_2d(snap, [f / 1e9], ang, geometry_units='meters')
    assert [s['polarization'] for s in r64['samples']][:1] == ['VV']
    for pol in ('TE', 'TM'):
        o = P.solve(k, [v], ang, pol)
        exp = 'VV' if pol == 'TE' else 'HH'
        a64 = np.array([complex(s['rcs_amp_real'], s['rcs_amp_imag']) for s in r64['samples'] if s['polarization'] == exp])
        s64 = np.array([s['rcs_linear'] for s in r64['samples'] if s['polarization'] == exp])
        s32 = np.array([s['rcs_linear'] for s in r32['samples'] if s['polarization'] == exp])
        assert np.max(np.abs(a64 - o['amplitude'])) <= 1e-9 * np.max(np.abs(o['amplitude']))
        db64 = 10 * np.log10(s64)
        mask = db64 > db64.max() - 40
        assert np.max(np.abs(10 * np.log10(s32 / s64))[mask]) <= 0.05


def test_concurrent_channels_match_single_channel_solves(ctx):
    """The co-polarised solve runs VV and HH on two device workers at once; each channel's
    result equals the same channel solved alone (the kernels are deterministic)."""
    from grim_20261007_b200.execution import linear_precision
    from grim_20261007_b200.twod.solver import (solve_monostatic_rcs_2d,
                                                solve_monostatic_rcs_2d_single_polarization)
    v, k, f, _ = S.airfoil_case(3, 640)
    snap = S.snapshot_from_polygons([v])
    ang = list(np.arange(0.0, 360.0, 1.5))
    for prec in ('double', 'mixed'):
        with linear_precision(prec):
            both = solve_monostatic_rcs_2d(snap, [f / 1e9], ang, geometry_units='meters', strict_quality_gate=False)
            for pol, exp in (('TE', 'VV'), ('TM', 'HH')):
                alone = solve_monostatic_rcs_2d_single_polarization(snap, [f / 1e9], ang, pol, geometry_units='meters',
                                                                    strict_quality_gate=False)
                a1 = np.array([complex(s['rcs_amp_real'], s['rcs_amp_imag']) for s in alone['samples']])
                a2 = np.array([complex(s['rcs_amp_real'], s['rcs_amp_imag']) for s in both['samples']
                               if s['polarization'] == exp])
                np.testing.assert_allclose(a2, a1, rtol=1e-13, atol=1e-13 * np.max(np.abs(a1)))


@pytest.mark.parametrize('grouped', ['1', '0'])
def test_frequency_sweep_pool_matches_single_frequency_solves(ctx, grouped, monkeypatch):
    """Pulse-basis systems: a multi-frequency request factors them with one grouped LU
    (GRIM_GROUPED_SWEEP=1, the default) or each on the device worker pool (0); either way every
    frequency's samples equal a one-frequency solve, in request order."""
    monkeypatch.setenv('GRIM_GROUPED_SWEEP', grouped)
    monkeypatch.setenv('GRIM_2D_FORMULATION', 'pulse')
    from grim_20261007_b200.execution import linear_precision
    from grim_20261007_b200.twod.solver import solve_monostatic_rcs_2d_single_polarization as solve1
    v = S.naca_symmetric(0.1, 160)
    snap = S.snapshot_from_polygons([v])
    for sg in snap['segments']:
        sg['properties'][1] = '-10'  # automatic meshing: 10 panels per wavelength
    freqs = [0.9, 3.1, 1.7, 2.4, 0.6]
    ang = list(np.arange(0.0, 180.0, 3.0))
    with linear_precision('mixed'):
        swept = solve1(snap, freqs, ang, 'TM', geometry_units='meters', strict_quality_gate=False)
        assert [s['frequency_ghz'] for s in swept['samples'][::len(ang)]] == freqs
        for i, f in enumerate(freqs):
            one = solve1(snap, [f], ang, 'TM', geometry_units='meters', strict_quality_gate=False)
            a1 = np.array([complex(s['rcs_amp_real'], s['rcs_amp_imag']) for s in one['samples']])
            block = swept['samples'][i * len(ang):(i + 1) * len(ang)]
            a2 = np.array([complex(s['rcs_amp_real'], s['rcs_amp_imag']) for s in block])
            np.testing.assert_allclose(a2, a1, rtol=1e-13, atol=1e-13 * np.max(np.abs(a1)))
    counts = swept['metadata']
    assert counts['dense_gpu_solve_count'] == len(freqs) and counts['panel_count_max'] > counts['panel_count_min']
    assert counts['dense_grouped_factorization_count'] == (len(freqs) if grouped == '1' else 0)


def test_galerkin_frequency_sweep_matches_single_frequency_solves(ctx, monkeypatch):
    """Linear-Galerkin systems (the default formulation) pivot throughout, so a multi-frequency
    request solves each on the device worker pool, never grouped; every frequency's samples
    equal a one-frequency solve, in request order."""
    monkeypatch.delenv('GRIM_2D_FORMULATION', raising=False)
    from grim_20261007_b200.execution import linear_precision
    from grim_20261007_b200.twod.solver import solve_monostatic_rcs_2d_single_polarization as solve1
    v = S.naca_symmetric(0.1, 160)
    snap = S.snapshot_from_polygons([v])
    for sg in snap['segments']:
        sg['properties'][1] = '-10'
    freqs = [0.9, 2.4, 1.7]
    ang = list(np.arange(0.0, 180.0, 3.0))
    with linear_precision('mixed'):
        swept = solve1(snap, freqs, ang, 'TE', geometry_units='meters', strict_quality_gate=False)
        for i, f in enumerate(freqs):
            one = solve1(snap, [f], ang, 'TE', geometry_units='meters', strict_quality_gate=False)
            a1 = np.array([complex(s['rcs_amp_real'], s['rcs_amp_imag']) for s in one['samples']])
            block = swept['samples'][i * len(ang):(i + 1) * len(ang)]
            a2 = np.array([complex(s['rcs_amp_real'], s['rcs_amp_imag']) for s in block])
            np.testing.assert_allclose(a2, a1, rtol=1e-13, atol=1e-13 * np.max(np.abs(a1)))
    assert swept['metadata']['dense_grouped_factorization_count'] == 0
    assert swept['metadata']['dense_gpu_solve_count'] == len(freqs)


@pytest.mark.parametrize('formulation', ['pulse', 'galerkin'])
def test_certified_entry_publishes_the_refined_mesh(ctx, formulation, monkeypatch):
    """The certified production entry solves the base and refined meshes of both channels --
    pulse systems in one grouped factorization, linear-Galerkin ones (partial pivoting) each
    on the worker pool -- and publishes the refined result: equal to a plain solve of the
    refined snapshot, with the reference-shaped certificate; limits it cannot meet raise."""
    monkeypatch.setenv('GRIM_2D_FORMULATION', formulation)
    from grim_20261007_b200.twod import certify
    from grim_20261007_b200.twod.solver import solve_monostatic_rcs_2d, solve_monostatic_rcs_2d_certified
    th = -2.0 * np.pi * np.arange(200) / 200.0
    v = np.stack([np.cos(th), np.sin(th)], -1)  # the 200-vertex circle of radius 1 m (clockwise)
    snap = S.snapshot_from_polygons([v])
    for sg in snap['segments']:
        sg['properties'][1] = '-30'  # 30 panels per wavelength; refined: 45
    ang = list(np.arange(0.0, 180.0, 4.0))
    freqs = [0.55, 0.7]  # ka 11.5 and 14.7 (400 -> 600 and 600 -> 800 panels)
    res = solve_monostatic_rcs_2d_certified(snap, freqs, ang, geometry_units='meters')
    ref = solve_monostatic_rcs_2d(certify.scale_snapshot_panel_density(snap, 1.5), freqs, ang,
                                  geometry_units='meters', strict_quality_gate=False)
    a = np.array([complex(s['rcs_amp_real'], s['rcs_amp_imag']) for s in res['samples']])
    b = np.array([complex(s['rcs_amp_real'], s['rcs_amp_imag']) for s in ref['samples']])
    np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-12 * np.max(np.abs(b)))
    for export in ('VV', 'HH'):
        meta = res['metadata']['channels'][export]
        assert meta['mesh_convergence_certified'] and meta['published_mesh'] == 'fine'
        gates = meta['mesh_convergence']
        assert len(gates) == 2 and all(gt['passed'] for gt in gates)
        assert all(gt['fine_panel_count'] > gt['base_panel_count'] for gt in gates)
        assert meta['dense_grouped_factorization_count'] == (2 if formulation == 'pulse' else 0)
    with pytest.raises(ValueError, match='mesh convergence failed'):
        solve_monostatic_rcs_2d_certified(snap, [0.55], ang, geometry_units='meters',
                                          mesh_convergence_policy={'complex_max_limit': 1e-9})
