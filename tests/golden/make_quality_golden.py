"""Generate ``mesh_certification.json``: the reference's own mesh-convergence certification
(``runs/quality.py:166`` ``scale_snapshot_panel_density``, ``:219``
``validate_mesh_convergence_policy``, ``:265`` ``evaluate_mesh_convergence``) on seeded
synthetic inputs.

Run in the build container (the reference tree is not present on GPU machines):

    python tests/golden/make_quality_golden.py /root/reference

The reference package is imported from its tree without writing into it (no bytecode).
Inputs: two snapshots with explicit, per-wavelength and automatic panel densities refined by
two factors; sample lists of two frequencies x 37 angles whose refined amplitudes differ by a
small (passing) and a large (failing) seeded perturbation, with a deep null.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def samples(amps, freqs, angles):
    out = []
    for fi, f in enumerate(freqs):
        for ai, a in enumerate(angles):
            z = complex(amps[fi, ai])
            lin = 0.25 * abs(z) ** 2
            out.append({'frequency_ghz': f, 'theta_inc_deg': a, 'theta_scat_deg': a, 'rcs_amp_real': z.real,
                        'rcs_amp_imag': z.imag, 'rcs_linear': lin,
                        'rcs_db': 10.0 * np.log10(max(lin, 1e-12))})
    return out


def cases():
    rng = np.random.default_rng(20261204)
    freqs = [1.25, 3.5]
    angles = [float(a) for a in np.arange(0.0, 181.0, 5.0)]
    base = rng.standard_normal((2, len(angles))) + 1j * rng.standard_normal((2, len(angles)))
    base[0, 7] = 1e-6 * (1 + 1j)  # a deep null
    small = base * (1 + 0.004 * (rng.standard_normal(base.shape) + 1j * rng.standard_normal(base.shape)))
    large = base * (1 + 0.2 * (rng.standard_normal(base.shape) + 1j * rng.standard_normal(base.shape)))
    return samples(base, freqs, angles), samples(small, freqs, angles), samples(large, freqs, angles)


def snapshot():
    segs = []
    for name, n in (('explicit', '7'), ('per_wavelength', '-12'), ('automatic', '0'), ('blank', '')):
        segs.append({'name': name, 'seg_type': '2', 'properties': ['2', n, '0', '0', '0'],
                     'point_pairs': [{'x1': 0.0, 'y1': 0.0, 'x2': 1.0, 'y2': 0.0}]})
    return {'segments': segs, 'ibcs': [], 'dielectrics': []}


def main(reference_root):
    sys.dont_write_bytecode = True
    sys.path.insert(0, os.path.join(reference_root, 'tools', 'GHOST'))
    from ghost_backend.runs import quality as Q
    base, small, large = cases()
    out = {'base': base, 'small': small, 'large': large, 'snapshot': snapshot(), 'scaled': {}, 'reports': {}}
    for factor in (1.5, 2.3):
        out['scaled'][str(factor)] = Q.scale_snapshot_panel_density(snapshot(), factor)
    out['policy_default'] = Q.validate_mesh_convergence_policy(None)
    for name, fine in (('small', small), ('large', large)):
        out['reports'][name] = Q.evaluate_mesh_convergence({'samples': base}, {'samples': fine}, rms_limit_db=1.0,
                                                          max_abs_limit_db=3.0)
    with open(os.path.join(HERE, 'mesh_certification.json'), 'w') as f:
        json.dump(out, f, indent=0, sort_keys=True)
    print('wrote mesh_certification.json', {k: out['reports'][k]['passed'] for k in out['reports']})


if __name__ == '__main__':
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get('GRIM_REFERENCE_ROOT', '/root/reference'))
