"""Generate ``ref_bor_modes.npz``: the reference body-of-revolution solver's own per-mode
operators and CFIE solves on seeded synthetic bodies.

Run in the build container (the reference tree is not present on GPU machines):

    python tests/golden/make_bor_golden.py /root/reference

The reference package is copied and its C kernels built exactly as ``make_golden.py``
does.  For each body the reference's ``BorPecSolver`` (``bor/solver.py:1324``, built by
``_prepared_surface``) gives, per signed mode m, the full node-based EFIE matrix
(``:1769`` ``assemble_mode``), the MFIE matrix (``:1962`` ``assemble_mfie_mode``) and the
tested plane-wave excitations (``:2462`` ``rhs_mode``, ``:2048`` ``rhs_mfie_mode``), and
``solve_bor`` (``:4066``) the CFIE far fields:

* ``sphere``: 12-element sphere, k = 2.5, modes -3..2 (table cap 4);
* ``graded``: 14-element closed body with cosine-spaced nodes (short elements near the
  poles, so pairs more than two elements apart fall inside the near gap), k = 4;
* ``sphere45``: the 45-element sphere at ka = 3 solved with ``formulation='cfie'``;
* ``resonant``: a 40-element sphere at ka = 2.7437, next to the first interior resonance
  (a zero of (x j_1(x))'), solved with the EFIE and the CFIE, with the Mie value.
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

MODES = (0, 1, -1, 2, -3)
ANGLES = (0.0, 35.0, 90.0, 150.0)


def sphere(n):
    t = np.linspace(0.0, math.pi, n + 1)
    return np.stack([np.sin(t), np.cos(t)], axis=1)


def graded(n):
    u = 0.5 * (1.0 - np.cos(np.linspace(0.0, math.pi, n + 1)))
    t = math.pi * u
    return np.stack([0.8 * np.sin(t) * (1.0 + 0.2 * np.cos(t)), 1.2 * np.cos(t)], axis=1)


def main(reference_root):
    sys.dont_write_bytecode = True
    from make_golden import _prepare
    _prepare(reference_root)
    from ghost_backend.bor import solver as BS
    from ghost_backend.validation import sphere as mie
    out = {'modes': np.array(MODES), 'angles': np.array(ANGLES)}
    for name, pts, k, mmax in (('sphere', sphere(12), 2.5, 4), ('graded', graded(14), 4.0, 4)):
        f = k * BS.C0 / (2.0 * math.pi)
        s = BS._prepared_surface(pts, f, gauss_order=3)
        out[f'{name}_points'] = pts
        out[f'{name}_k'] = np.array(s.k)
        out[f'{name}_mmax'] = np.array(mmax)
        for m in MODES:
            out[f'{name}_efie_{m}'] = s.assemble_mode(m, mmax)
            out[f'{name}_mfie_{m}'] = s.assemble_mfie_mode(m, mmax)
            for kind, fun in (('rhs', s.rhs_mode), ('rhs_mfie', s.rhs_mfie_mode)):
                out[f'{name}_{kind}_{m}'] = np.stack([np.stack([fun(m, a, pol) for a in ANGLES], axis=1)
                                                      for pol in ('VV', 'HH')])
    thetas = np.array([0.0, 30.0, 60.0, 90.0, 120.0, 150.0, 180.0])
    pts = sphere(45)
    f = 3.0 * BS.C0 / (2.0 * math.pi)
    r = BS.solve_bor(pts, f, thetas, formulation='cfie')
    out.update(sphere45_points=pts, sphere45_freq_hz=np.array(f), sphere45_thetas=thetas,
               sphere45_amp_vv=np.asarray(r['amp_vv']), sphere45_amp_hh=np.asarray(r['amp_hh']),
               sphere45_modes_used=np.array(int(r['modes_used'])))
    pts = sphere(40)
    f = 2.7437 * BS.C0 / (2.0 * math.pi)
    th = np.array([0.0, 90.0, 180.0])
    for form in ('efie', 'cfie'):
        r = BS.solve_bor(pts, f, th, formulation=form, n_modes=12)
        out[f'resonant_{form}_amp_vv'] = np.asarray(r['amp_vv'])
        out[f'resonant_{form}_amp_hh'] = np.asarray(r['amp_hh'])
    out.update(resonant_points=pts, resonant_freq_hz=np.array(f), resonant_thetas=th,
               resonant_mie_sigma=np.array(mie.sigma_pec_sphere(1.0, f)))
    np.savez_compressed(os.path.join(HERE, 'ref_bor_modes.npz'), **out)
    print('wrote ref_bor_modes.npz', len(out), 'arrays')


if __name__ == '__main__':
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get('GRIM_REFERENCE_ROOT', '/root/reference'))
