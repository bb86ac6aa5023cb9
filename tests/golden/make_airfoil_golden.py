"""Reference-solver amplitudes on the seeded NACA airfoil of the headline workload.

Run in the build container (the reference tree is not present on GPU machines):

    python tests/golden/make_airfoil_golden.py [reference_root]

The reference is copied to a writable temporary folder and its C kernels are built from
their own sources (``make_golden._prepare``; the shipped ``.dll`` files are never used).
For ``synthetic.airfoil_case(seed=0, n)`` (NACA 00tt, blunt trailing edge, cosine
spacing, lambda / 10 on average) at n = 256, 1024 and 2048 it calls the reference's
``solve_monostatic_rcs_2d_single_polarization(snapshot, [f], angles, pol,
geometry_units='meters', strict_quality_gate=False, solver_method='direct')``
(``twod/solver.py:1988``) for TM and TE at the headline's 720 angles (0.5 degree steps)
and stores the complex stored amplitudes B and sigma_2D in ``ref_airfoil.npz``; the
reference's own stage seconds are printed.
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
SIZES = (256, 1024, 2048)


def main(reference_root):
    sys.dont_write_bytecode = True
    sys.path.insert(0, HERE)
    sys.path.insert(0, ROOT)
    from make_golden import _prepare
    _prepare(reference_root)
    import ghost_backend.twod.solver as rcs
    from grim_20261007_b200 import synthetic as S
    angles = [0.5 * i for i in range(720)]
    out = {'angles': np.array(angles), 'sizes': np.array(SIZES)}
    for n in SIZES:
        v, k, f_hz, t = S.airfoil_case(0, n)
        snap = S.snapshot_from_polygons([v])
        out[f'n{n}_k'] = k
        out[f'n{n}_frequency_ghz'] = f_hz / 1e9
        out[f'n{n}_thickness'] = t
        for pol in ('TM', 'TE'):
            t0 = time.perf_counter()
            res = rcs.solve_monostatic_rcs_2d_single_polarization(
                snap, [f_hz / 1e9], angles, pol, geometry_units='meters', strict_quality_gate=False,
                solver_method='direct', max_panels=20000)
            s = res['samples']
            out[f'n{n}_amp_{pol}'] = np.array([complex(r['rcs_amp_real'], r['rcs_amp_imag']) for r in s])
            out[f'n{n}_sigma_{pol}'] = np.array([r['rcs_linear'] for r in s])
            stages = res['metadata'].get('runtime_profile', {}).get('stage_seconds', {})
            print(f'n={n} {pol}: {time.perf_counter() - t0:.1f} s, stages {stages}', flush=True)
    np.savez_compressed(os.path.join(HERE, 'ref_airfoil.npz'), **out)
    print('wrote', os.path.join(HERE, 'ref_airfoil.npz'))


if __name__ == '__main__':
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get('GRIM_REFERENCE_ROOT', '/root/reference'))
