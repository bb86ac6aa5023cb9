"""Host-side logic and the C ABI library, without a GPU."""
import ctypes
import math

import numpy as np
import pytest

from grim_20261007_b200 import _lib, synthetic as S
from grim_20261007_b200.twod import geometry as geo
from oracle import pulse2d as P


def test_library_loads_and_exports_every_declared_symbol():
    lib = _lib.load()
    declared = _lib.header_symbols()
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(lib, name), name
    bound = {s[0] for s in _lib.SIGNATURES}
    assert set(declared) <= bound
    assert lib.grim_version() >= 1


def test_cond_system_struct_matches_the_c_layout(tmp_path):
    """_lib.GrimCondSystem has grim_cond_system's size and field offsets (compiled here
    against include/grimgpu.h)."""
    import os
    import shutil
    import subprocess
    cc = shutil.which('gcc') or shutil.which('cc')
    if cc is None:
        pytest.skip('no C compiler')
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), 'include')
    fields = [f[0] for f in _lib.GrimCondSystem._fields_]
    src = tmp_path / 'layout.c'
    body = ''.join(f'    printf("%zu\\n", offsetof(grim_cond_system, {f}));\n' for f in fields)
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "grimgpu.h"\nint main(void) {\n'
                   '    printf("%zu\\n", sizeof(grim_cond_system));\n' + body + '    return 0;\n}\n')
    exe = tmp_path / 'layout'
    subprocess.run([cc, '-I', inc, str(src), '-o', str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    want = [ctypes.sizeof(_lib.GrimCondSystem)] + [getattr(_lib.GrimCondSystem, f).offset for f in fields]
    assert got == want


def test_library_reports_errors_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip('a GPU is present')
    lib = _lib.load()
    h = ctypes.c_void_p()
    status = lib.grim_create(0, ctypes.byref(h))
    assert status != _lib.GRIM_OK
    assert _lib.last_error()
    assert lib.grim_fill2d(None, 0, 10, None, None, 1.0, None, 10, 0) == _lib.GRIM_ERR_ARGUMENT


def test_snapshot_panel_rules():
    v = S.circle(1.0, 12)
    snap = S.snapshot_from_polygons([v])
    polys = geo.contours_from_snapshot(snap, 'meters')
    assert len(polys) == 1 and polys[0].shape == (12, 2)
    np.testing.assert_allclose(polys[0], v, atol=1e-15)
    # N = 3 panels per primitive
    for seg in snap['segments']:
        seg['properties'][1] = '3'
    assert geo.contours_from_snapshot(snap, 'meters')[0].shape == (36, 2)
    # N < 0: |N| panels per wavelength
    for seg in snap['segments']:
        seg['properties'][1] = '-10'
    side = 2 * math.sin(math.pi / 12)
    got = geo.contours_from_snapshot(snap, 'meters', wavelength=0.1)[0].shape[0]
    assert got == 12 * math.ceil(side * 10 / 0.1)
    # inches
    for seg in snap['segments']:
        seg['properties'][1] = '1'
    np.testing.assert_allclose(geo.contours_from_snapshot(snap, 'inches')[0], v * 0.0254)


def test_snapshot_rejects_out_of_scope_boundaries():
    snap = S.snapshot_from_polygons([S.circle(1.0, 8)])
    snap['segments'][0]['seg_type'] = 3
    with pytest.raises(NotImplementedError):
        geo.contours_from_snapshot(snap, 'meters')
    snap = S.snapshot_from_polygons([S.circle(1.0, 8)])
    snap['dielectrics'] = [['1', '4', '0', '1', '0']]
    with pytest.raises(NotImplementedError):
        geo.contours_from_snapshot(snap, 'meters')


def test_panel_geometry_matches_oracle_and_normals_point_outward():
    v = S.naca_symmetric(0.12, 64)
    g = geo.panel_geometry([v])
    c, t, h, n = P.panel_arrays([v])
    np.testing.assert_array_equal(g[:, 0:2], c)
    np.testing.assert_array_equal(g[:, 2:4], t)
    np.testing.assert_array_equal(g[:, 4], h)
    np.testing.assert_array_equal(g[:, 5:7], n)
    # outward: centroid-to-midpoint has positive projection on the normal for a convex-ish body
    cen = v.mean(axis=0)
    assert np.mean(np.sum((c - cen) * n, axis=1) > 0) > 0.95
    # counter-clockwise input gives the same outward normals
    g2 = geo.panel_geometry([v[::-1]])
    assert np.allclose(np.sort(g2[:, 5]), np.sort(g[:, 5]))
    np.testing.assert_array_equal(geo.te_curvature_correction([v]), P.te_curvature_correction([v]))


def test_te_curvature_correction_on_circle():
    n = 50
    corr = geo.te_curvature_correction([S.circle(2.0, n)])
    side = 2 * 2.0 * math.sin(math.pi / n)
    kappa = (2 * math.pi / n) / side
    np.testing.assert_allclose(corr, kappa * side / (4 * math.pi), rtol=1e-12)


def test_synthetic_workloads_are_seeded_and_clockwise():
    v1, k1, f1, t1 = S.airfoil_case(7, 2048)
    v2, k2, f2, t2 = S.airfoil_case(7, 2048)
    np.testing.assert_array_equal(v1, v2)
    assert 0.08 <= t1 <= 0.15 and v1.shape == (2048, 2)
    b = np.roll(v1, -1, axis=0)
    area = 0.5 * np.sum(v1[:, 0] * b[:, 1] - b[:, 0] * v1[:, 1])
    assert area < 0
    lam = 2 * math.pi / k1
    assert abs(geo.perimeter([v1]) / 2048 - lam / 10) < 1e-12
    gen, length, half = S.ogive_case(3)
    assert gen[0, 0] == 0 and gen[-1, 0] == 0 and gen[0, 1] > gen[-1, 1]
    assert 2 <= length <= 4 and 15 <= half <= 30


def test_airfoil_sweep_case_sizes():
    from grim_20261007_b200 import synthetic as S
    cases, t = S.airfoil_sweep_case(3, 256)
    ns = [len(v) for v, _k, _f in cases]
    fs = [f for _v, _k, f in cases]
    assert len(cases) == 256 and all(n % 2 == 0 for n in ns)
    assert max(ns) == 4096 and min(ns) >= 64
    assert abs(fs[-1] / fs[0] - 20.0) < 1e-9 and all(b > a for a, b in zip(fs, fs[1:]))
    assert ns == sorted(ns)


def test_tuning_buckets_and_cache_roundtrip(tmp_path, monkeypatch):
    from grim_20261007_b200 import tuning
    assert tuning.bucket(2048, 720) == (2048, 1024)
    assert tuning.bucket(100, 1) == (512, 16)
    assert tuning.bucket(2049, 1024) == (2560, 1024)
    monkeypatch.setenv('GRIM_TUNING_CACHE', str(tmp_path / 'tuning.json'))
    monkeypatch.setattr(tuning, '_table', None)
    assert tuning.lookup('dev', 2048, 720) is None
    tuning._store(tuning._key('dev', 2048, 720), {'choice': {'solve_bn': 64, 'gs_block': 512}})
    monkeypatch.setattr(tuning, '_table', None)  # a fresh process reads the file
    assert tuning.lookup('dev', 2000, 600)['choice'] == {'solve_bn': 64, 'gs_block': 512}


def test_cpu_dense_backend_is_refused_not_run_on_the_gpu(monkeypatch):
    from grim_20261007_b200 import synthetic as S
    from grim_20261007_b200.execution import require_gpu_dense_backend
    from grim_20261007_b200.twod import solver
    monkeypatch.setenv('GHOST_DENSE_BACKEND', 'cpu')
    with pytest.raises(RuntimeError, match='CPU solver'):
        require_gpu_dense_backend()
    snap = S.snapshot_from_polygons([S.circle(1.0, 32)])
    with pytest.raises(RuntimeError, match='CPU solver'):
        solver.solve_monostatic_rcs_2d_single_polarization(snap, [0.3], [0.0], 'TM', geometry_units='meters')
    monkeypatch.setenv('GHOST_DENSE_BACKEND', 'auto')
    assert require_gpu_dense_backend() == 'auto'


def _snap(polys):
    return S.snapshot_from_polygons(polys)


def test_geometry_validation_rejects_what_the_reference_rejects():
    """The reference's fatal solver-side checks (twod/geometry.py:1121-1457, geometry/io.py:712)
    restated: the sharp-trailing-edge airfoil at 2048 elements is a crack (its upper and lower
    vertices next to the tip are 7e-7 m apart), the blunt one is accepted; duplicate,
    crossing and wrongly wound contours are refused."""
    t = 0.12458731811250179
    with pytest.raises(ValueError, match='Geometry crack'):
        geo.contours_from_snapshot(_snap([S.naca_symmetric(t, 2048, closed_te=True)]), 'meters')
    polys = geo.contours_from_snapshot(_snap([S.naca_symmetric(t, 2048)]), 'meters')
    assert len(polys) == 1 and len(polys[0]) == 2048
    geo.contours_from_snapshot(_snap([S.naca_symmetric(t, 1024, closed_te=True)]), 'meters')  # as the reference
    with pytest.raises(ValueError, match='orientation'):
        geo.contours_from_snapshot(_snap([S.circle(1.0, 40)[::-1]]), 'meters')
    # a body inside a void inside a body: the void runs counter-clockwise
    geo.contours_from_snapshot(_snap([S.circle(2.0, 60), S.circle(1.0, 40)[::-1], S.circle(0.5, 30)]), 'meters')
    with pytest.raises(ValueError, match='Duplicate primitive'):
        geo.contours_from_snapshot(_snap([S.circle(1.0, 40), S.circle(1.0, 40)]), 'meters')
    bow = np.array([[0.0, 0.0], [1.0, 1.0], [1.0, 0.0], [0.0, 1.0]])
    with pytest.raises(ValueError, match='intersection'):
        geo.contours_from_snapshot(_snap([bow]), 'meters')
    with pytest.raises(ValueError, match='Collinear overlapping'):
        geo.contours_from_snapshot(_snap([np.array([[0.0, 0.0], [0.0, 1.0], [1.0, 1.0], [1.0, 0.0], [0.5, 0.0],
                                                     [0.7, 0.0]])]), 'meters')
    snap = _snap([S.circle(1.0, 40)])
    snap['segments'][0]['point_pairs'][5]['x2'] += 1e-3
    with pytest.raises(ValueError, match='disconnected primitive chain'):
        geo.contours_from_snapshot(snap, 'meters')


def test_geometry_validation_is_cheap_on_the_headline_airfoil():
    import time
    snap = _snap([S.airfoil_case(0, 2048)[0]])
    geo.contours_from_snapshot(snap, 'meters')
    t0 = time.perf_counter()
    geo.contours_from_snapshot(snap, 'meters')
    assert time.perf_counter() - t0 < 0.05


def test_public_solve_raises_the_geometry_error_checked_beside_the_solve(monkeypatch):
    """The reference's geometry checks run on a host thread while the systems are solved; a
    rejected geometry still raises its ValueError from the public entry (before any result),
    even when the solve itself fails on that geometry, and a valid one returns normally."""
    from grim_20261007_b200.twod import solver

    class _Ctx:
        device_name = 'fake'

    calls = []

    def fake_solve(meshes, f, elevs, pol, precision, abort_event, condition=False):
        calls.append((pol, f))
        if fail['now']:
            raise RuntimeError('solve failed')
        samples = [{'frequency_ghz': f, 'theta_inc_deg': e, 'theta_scat_deg': e, 'rcs_linear': 1.0, 'rcs_db': 0.0,
                    'rcs_amp_real': 1.0, 'rcs_amp_imag': 0.0, 'rcs_amp_phase_deg': 0.0, 'linear_residual': 1e-15}
                   for e in elevs]
        return dict(samples=samples, residuals=[1e-15] * len(elevs), event={'used': 'gpu_grim', 'n': 8}, n=8,
                    seconds=0.0, condition_est=None)

    fail = {'now': False}
    monkeypatch.setenv('GRIM_SWEEP_WORKERS', '1')
    monkeypatch.setenv('GRIM_GROUPED_SWEEP', '0')
    monkeypatch.setattr(solver, '_solve_frequency', fake_solve)
    monkeypatch.setattr(solver, 'require_cuda', lambda: None)
    monkeypatch.setattr(solver, 'context', lambda: _Ctx())
    t = 0.12458731811250179
    cracked = _snap([S.naca_symmetric(t, 2048, closed_te=True)])
    for failing in (False, True):
        fail['now'] = failing
        with pytest.raises(ValueError, match='Geometry crack'):
            solver.solve_monostatic_rcs_2d_single_polarization(cracked, [1.0], [0.0, 10.0], 'TM',
                                                               geometry_units='meters')
    fail['now'] = False
    good = solver.solve_monostatic_rcs_2d_single_polarization(_snap([S.naca_symmetric(t, 2048)]), [1.0, 2.0],
                                                              [0.0, 10.0], 'TM', geometry_units='meters')
    assert len(good['samples']) == 4 and ('TM', 2.0) in calls
