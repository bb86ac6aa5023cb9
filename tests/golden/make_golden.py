"""Generate the golden fixtures in this folder by running the reference itself.

Run in the build container (the reference tree is not present on GPU machines):

    python tests/golden/make_golden.py /root/reference

The reference package is copied to a temporary writable folder (its tree is
read-only and it writes bytecode and native builds next to its sources), its
C kernels are built from their own sources with its own build scripts, and then:

* ``mie_cylinder.npz``  -- ``validation/cylinder.py:37`` complex amplitudes B and
  ``:68`` sigma_2D for a grid of ka, both polarisations;
* ``mie_sphere.npz``    -- ``validation/sphere.py:196`` PEC sphere sigma for a grid of ka;
* ``ref_cylinder_c1.npz`` -- the reference solver
  (``twod/solver.py:1988`` ``solve_monostatic_rcs_2d_single_polarization``,
  ``solver_method='direct'``) on the 200-panel a = 1 m cylinder at ka = 10,
  360 angles, TM and TE: complex stored amplitudes B and sigma_2D;
* ``ref_dense_system.npz`` -- the reference's own assembled dense systems as they
  arrive at its GPU hook (``twod/solver.py:355`` ``_solve_dense_gpu(a_eval, rhs_eval)``),
  captured with ``GHOST_DENSE_BACKEND=gpu`` and a patched hook exactly as
  ``tests/test_rcs_physics_regression.py:338-365`` does, together with the
  reference CPU solution (LAPACK getrf/getrs via ``linalg/dense.py``) and the
  2x2 system from that test.
* ``ref_bor_sphere.npz`` -- the reference body-of-revolution solver
  (``bor/solver.py:4066`` ``solve_bor``) on a PEC sphere, with the Mie value.
"""
from __future__ import annotations

import math
import os
import shutil
import subprocess
import sys
import tempfile
from unittest import mock

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _prepare(reference_root):
    work = tempfile.mkdtemp(prefix='ghost_ref_')
    src = os.path.join(reference_root, 'tools', 'GHOST')
    dst = os.path.join(work, 'GHOST')
    shutil.copytree(src, dst, ignore=shutil.ignore_patterns('*.dll'))
    for root, dirs, files in os.walk(dst):
        os.chmod(root, 0o755)
        for f in files:
            os.chmod(os.path.join(root, f), 0o644)
    env = dict(os.environ, PYTHONDONTWRITEBYTECODE='1')
    for script in ('ghost_backend/twod/assembly/native/build.py', 'ghost_backend/bor/native/build_kernel.py'):
        subprocess.run([sys.executable, script], cwd=dst, env=env, check=True,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    sys.path.insert(0, dst)
    return dst


def circle_snapshot(radius, count):
    theta = np.linspace(0.0, -2.0 * np.pi, count + 1)
    pairs = [dict(x1=float(radius * np.cos(theta[i])), y1=float(radius * np.sin(theta[i])),
                  x2=float(radius * np.cos(theta[i + 1])), y2=float(radius * np.sin(theta[i + 1])))
             for i in range(count)]
    seg = dict(name='circle', seg_type=2, properties=['2', '1', '0', '0', '0'], point_pairs=pairs)
    return dict(segments=[seg], ibcs=[], dielectrics=[])


def main(reference_root):
    sys.dont_write_bytecode = True
    _prepare(reference_root)
    from ghost_backend.validation import cylinder, sphere
    import ghost_backend.twod.solver as rcs

    # --- Mie (cylinder / sphere) -------------------------------------------------
    ka = np.array([0.5, 1.0, 2.404825557695773, 5.0, 10.0, 25.0])
    amps = np.zeros((2, len(ka)), complex)
    sig = np.zeros((2, len(ka)))
    for i, x in enumerate(ka):
        f = x * cylinder.C0 / (2 * math.pi * 1.0)
        for p, pol in enumerate(('TM', 'TE')):
            amps[p, i] = cylinder.pec_cylinder_backscatter_amplitude(1.0, f, pol)
            sig[p, i] = cylinder.sigma_pec_cylinder(1.0, f, pol)
    np.savez(os.path.join(HERE, 'mie_cylinder.npz'), ka=ka, radius=1.0, c0=cylinder.C0,
             amplitude=amps, sigma=sig, pols=np.array(['TM', 'TE']))
    ka_s = np.array([0.5, 1.0, 3.0, 5.0, 10.0, 20.0])
    sig_s = np.array([sphere.sigma_pec_sphere(1.0, x * sphere.C0 / (2 * math.pi)) for x in ka_s])
    np.savez(os.path.join(HERE, 'mie_sphere.npz'), ka=ka_s, radius=1.0, c0=sphere.C0, sigma=sig_s)

    # --- reference solver at the 200-panel cylinder, ka = 10 --------------------
    k = 10.0
    f_ghz = k * rcs.C0 / (2 * math.pi) / 1e9
    angles = [float(a) for a in range(360)]
    snap = circle_snapshot(1.0, 200)
    out = {}
    for pol in ('TM', 'TE'):
        res = rcs.solve_monostatic_rcs_2d_single_polarization(
            snap, [f_ghz], angles, pol, geometry_units='meters', strict_quality_gate=False,
            solver_method='direct', max_panels=1000)
        s = res['samples']
        out['amp_' + pol] = np.array([complex(r['rcs_amp_real'], r['rcs_amp_imag']) for r in s])
        out['sigma_' + pol] = np.array([r['rcs_linear'] for r in s])
        out['db_' + pol] = np.array([r['rcs_db'] for r in s])
    np.savez(os.path.join(HERE, 'ref_cylinder_c1.npz'), k=k, radius=1.0, n_panels=200,
             frequency_ghz=f_ghz, angles=np.array(angles), **out)

    # --- reference dense systems at the GPU hook --------------------------------
    captured = []

    def fake_gpu(a_eval, rhs_eval):
        captured.append((np.array(a_eval), np.array(rhs_eval)))
        return np.linalg.solve(a_eval, rhs_eval), 'capture'

    systems = {}
    cases = [('cyl64_ka1', 0.1, 64, 1.0), ('cyl64_ka2p4', 0.1, 64, 2.404825557695773), ('cyl96_ka5', 0.1, 96, 5.0)]
    for name, radius, count, kav in cases:
        freq = kav * rcs.C0 / (2 * math.pi * radius) / 1e9
        for pol in ('TM', 'TE'):
            captured.clear()
            with mock.patch.dict(os.environ, {rcs.DENSE_GPU_BACKEND_ENV: 'gpu'}), \
                    mock.patch.object(rcs, '_solve_dense_gpu', side_effect=fake_gpu):
                rcs.solve_monostatic_rcs_2d_single_polarization(
                    circle_snapshot(radius, count), [freq], [0.0, 30.0, 90.0, 135.0, 200.0, 300.0], pol,
                    geometry_units='meters', strict_quality_gate=False, solver_method='direct', max_panels=1000)
            a_eval, rhs_eval = captured[0]
            import scipy.linalg as sla
            x = sla.lu_solve(sla.lu_factor(a_eval), rhs_eval)
            systems[f'{name}_{pol}_a'] = a_eval
            systems[f'{name}_{pol}_b'] = rhs_eval
            systems[f'{name}_{pol}_x'] = x
    systems['tiny_a'] = np.asarray([[4.0 + 0.2j, 1.0], [1.0, 3.0 - 0.1j]], dtype=np.complex128)
    systems['tiny_b'] = np.asarray([[1.0 + 0.5j], [-0.2j]], dtype=np.complex128)
    systems['tiny_x'] = np.linalg.solve(systems['tiny_a'], systems['tiny_b'])
    np.savez_compressed(os.path.join(HERE, 'ref_dense_system.npz'), **systems)

    # --- reference body-of-revolution solver on a PEC sphere --------------------
    from ghost_backend.bor.solver import solve_bor
    n_el = 45
    t = np.linspace(0.0, math.pi, n_el + 1)
    pts = np.stack([np.sin(t), np.cos(t)], axis=1)  # (rho, z), +z axis to -z axis
    ka_b = 3.0
    freq_hz = ka_b * sphere.C0 / (2 * math.pi)
    thetas = np.array([0.0, 30.0, 60.0, 90.0, 120.0, 150.0, 180.0])
    res = solve_bor(pts, freq_hz, thetas, formulation='efie')
    res_c = solve_bor(pts, freq_hz, thetas)
    np.savez(os.path.join(HERE, 'ref_bor_sphere.npz'), points=pts, freq_hz=freq_hz, thetas=thetas,
             sigma_vv_efie=np.asarray(res['sigma_vv']), sigma_hh_efie=np.asarray(res['sigma_hh']),
             amp_vv_efie=np.asarray(res['amp_vv']), amp_hh_efie=np.asarray(res['amp_hh']),
             sigma_vv_cfie=np.asarray(res_c['sigma_vv']), sigma_hh_cfie=np.asarray(res_c['sigma_hh']),
             amp_vv_cfie=np.asarray(res_c['amp_vv']), amp_hh_cfie=np.asarray(res_c['amp_hh']),
             modes_used=int(res['modes_used']), n_unknowns=int(res['n_unknowns']),
             mie_sigma=sphere.sigma_pec_sphere(1.0, freq_hz))
    print('golden fixtures written to', HERE)


if __name__ == '__main__':
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get('GRIM_REFERENCE_ROOT', '/root/reference'))
