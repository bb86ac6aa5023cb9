"""Generate ``tests/golden/grim/*.grim``: the reference's own ``.grim`` archives
(``io/grim.py:1034`` ``export_result_to_grim``, format versions 1 and 2) of the seeded
result dicts of ``results()`` (recreated by the tests, not stored): a single-polarisation
TM result with a repeated sample and metadata holding non-finite, complex and nested
values, a co-polarised VV/HH result in the reference's merged shape, and the same
single-polarisation result exported without its raw complex amplitudes.

Run in the build container (the reference tree is not present on GPU machines):

    python tests/golden/make_grim_golden.py <reference root>

(or with the root in GRIM_REFERENCE_ROOT).  The reference package is imported from its tree
without writing into it (no bytecode).
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, 'grim')
C0 = 299_792_458.0


def _rows(rng, freqs, angles, pol=None, internal=None):
    rows = []
    for f in freqs:
        k = 2.0 * math.pi * f * 1e9 / C0
        for a in angles:
            amp = complex(rng.standard_normal(), rng.standard_normal()) * 10.0 ** rng.uniform(-2, 1)
            lin = abs(amp) ** 2 / (4.0 * k)
            row = {'frequency_ghz': f, 'theta_inc_deg': a, 'theta_scat_deg': a, 'rcs_linear': lin,
                   'rcs_db': 10.0 * math.log10(max(lin, 1e-12)), 'rcs_amp_real': amp.real, 'rcs_amp_imag': amp.imag,
                   'rcs_amp_phase_deg': math.degrees(math.atan2(amp.imag, amp.real)),
                   'linear_residual': float(10.0 ** rng.uniform(-15, -12))}
            if pol is not None:
                row['polarization'] = pol
                row['polarization_internal'] = internal
            rows.append(row)
    return rows


def results():
    """name -> (result dict, export keyword arguments)."""
    rng = np.random.default_rng(20261204)
    freqs = [1.5, 3.0]
    angles = [0.0, 30.0, 45.5, 90.0, 180.0, 270.25]
    single = _rows(rng, freqs, angles)
    # a repeated coordinate with the same values: its power is made exactly representable in
    # float32 (the reference compares a repeat with the float32-stored first sample to 1e-12)
    row = single[3]
    target = float(np.float32(row['rcs_linear']))
    scale = math.sqrt(target / row['rcs_linear'])
    row.update(rcs_linear=target, rcs_amp_real=row['rcs_amp_real'] * scale, rcs_amp_imag=row['rcs_amp_imag'] * scale)
    single.append(dict(row))
    meta = {'residual_norm_max': 1e-13, 'condition_est_max': float('nan'), 'ratio': float('inf'),
            'z': complex(1.0, -2.0), 'nested': {'b': [1, 2.5, None], 'a': 'text'}, 'count': np.int64(3),
            'quality_gate': {'passed': True, 'reason': 'ok'}}
    res_tm = {'solver': '2d_bie_mom_rcs', 'scattering_mode': 'monostatic',
              'amplitude_convention': 'A_physical_asymptotic = +j * B_stored', 'amplitude_version': 2,
              'polarization': 'TM', 'polarization_export': 'TM', 'samples': single, 'metadata': meta}
    vv = _rows(rng, freqs, angles, 'VV', 'TE')
    hh = _rows(rng, freqs, angles, 'HH', 'TM')
    merged = []
    for a, b in zip(vv, hh):
        merged += [a, b]
    res_co = {'solver': '2d_bie_mom_rcs', 'scattering_mode': 'monostatic',
              'amplitude_convention': 'A_physical_asymptotic = +j * B_stored', 'amplitude_version': 2,
              'rcs_log_unit': 'dBke', 'rcs_linear_quantity': 'sigma_2d', 'polarizations': ['VV', 'HH'],
              'polarization_mapping': {'VV': 'TE', 'HH': 'TM'}, 'samples': merged,
              'co_solved_samples': {'VV': vv, 'HH': hh},
              'metadata': {'polarizations': ['VV', 'HH'], 'residual_norm_max': 2e-13}}
    return {
        'tm': (res_tm, {'source_path': 'airfoil.json', 'history': 'seeded'}),
        'co': (res_co, {'source_path': '', 'history': ''}),
        'tm_noraw': (res_tm, {'source_path': 'airfoil.json', 'history': 'seeded',
                              'preserve_raw_complex_amplitude': False}),
    }


def main(reference_root):
    sys.dont_write_bytecode = True
    sys.path.insert(0, os.path.join(reference_root, 'tools', 'GHOST'))
    from ghost_backend.io.grim import export_result_to_grim
    os.makedirs(OUT, exist_ok=True)
    for name, (res, kw) in results().items():
        for version in (1, 2):
            export_result_to_grim(res, os.path.join(OUT, f'{name}_v{version}.grim'), format_version=version, **kw)


if __name__ == '__main__':
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('GRIM_REFERENCE_ROOT')
    if not root:
        raise SystemExit('usage: make_grim_golden.py <reference root> (or GRIM_REFERENCE_ROOT)')
    main(root)
