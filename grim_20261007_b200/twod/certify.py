"""Mesh-convergence certification of 2-D results (base and refined mesh), the reference's
production path ``twod/solver.py:3663-3880`` (``_run_certified_2d_pair``,
``_certify_2d_results``) with the policy and metrics of ``runs/quality.py:23-547``.

The result of a certified solve is the refined-mesh result, published only when it agrees
with the base-mesh result within the policy's limits: the primary metric is the complex
far-field change normalised by each frequency's peak amplitude (defined at nulls too); dB
changes are taken on ``20 log10(|A| + floor * peak)`` and phase changes only where both
meshes are above ``floor * peak``.  The same formulas and limits are kept here so that a
result certified by one code is certified by the other; the GPU side solves every base and
refined system of a request in one grouped factorization (``twod/solver.py``).
"""
from __future__ import annotations

import copy
import math

import numpy as np

LEVEL_FLOOR = 3.0e-2  # runs/quality.py:23, -30 dB below the per-frequency peak
EPS = 1e-12
DEFAULT_PANELS_PER_WAVELENGTH = 20

PRODUCTION_DEFAULTS = {  # runs/quality.py:25-35
    'fine_factor': 1.5,
    'rms_limit_db': 1.0,
    'max_abs_limit_db': 3.0,
    'complex_rms_limit': 0.02,
    'complex_max_limit': 0.05,
    'phase_rms_limit_deg': 5.0,
    'phase_max_limit_deg': 15.0,
    'phase_floor_relative': LEVEL_FLOOR,
    'db_floor_relative': LEVEL_FLOOR,
}


def validate_policy(policy=None):
    """Complete, finite policy (runs/quality.py:219-262): unknown fields and out-of-range
    values raise ValueError."""
    supplied = dict(policy or {})
    unknown = sorted(set(supplied) - set(PRODUCTION_DEFAULTS))
    if unknown:
        raise ValueError('Unknown mesh convergence policy field(s): ' + ', '.join(unknown))
    out = dict(PRODUCTION_DEFAULTS)
    out.update(supplied)
    for name, raw in list(out.items()):
        try:
            value = float(raw)
        except (TypeError, ValueError, OverflowError) as exc:
            raise ValueError(f'{name} must be a finite number.') from exc
        if not math.isfinite(value):
            raise ValueError(f'{name} must be a finite number.')
        out[name] = value
    if out['fine_factor'] <= 1.0:
        raise ValueError('fine_factor must be > 1.0.')
    for name in ('rms_limit_db', 'max_abs_limit_db', 'complex_rms_limit', 'complex_max_limit',
                 'phase_rms_limit_deg', 'phase_max_limit_deg'):
        if out[name] < 0.0:
            raise ValueError(f'{name} must be nonnegative.')
    for name in ('phase_floor_relative', 'db_floor_relative'):
        if not 0.0 <= out[name] < 1.0:
            raise ValueError(f'{name} must be in [0, 1).')
    return out


def scale_snapshot_panel_density(snapshot, fine_factor):
    """Deep copy of the snapshot with every segment's panel-density property (properties[1])
    refined by ``fine_factor`` (runs/quality.py:166-216): N > 0 panels -> max(N + 1,
    ceil(N f)); N < 0 panels per wavelength -> -max(|N| + 1, ceil(|N| f)); 0 (automatic)
    -> -max(2, ceil(20 f))."""
    factor = float(fine_factor)
    if factor <= 1.0:
        raise ValueError('fine_factor must be > 1.0.')
    out = copy.deepcopy(snapshot)
    segments = list(out.get('segments', []) or [])
    for seg in segments:
        props = [str(p) for p in list(seg.get('properties', []) or [])]
        props += [''] * (6 - len(props))
        try:
            base_n = int(round(float(str(props[1]).strip() or 0)))
        except Exception:  # noqa: BLE001 - an unreadable density is the automatic one
            base_n = 0
        if base_n == 0:
            props[1] = str(-max(2, int(math.ceil(DEFAULT_PANELS_PER_WAVELENGTH * factor))))
        elif base_n > 0:
            props[1] = str(max(base_n + 1, int(math.ceil(base_n * factor))))
        else:
            ppw = abs(base_n)
            props[1] = str(-max(ppw + 1, int(math.ceil(ppw * factor))))
        seg['properties'] = props
        seg['seg_type'] = props[0] if props[0] else seg.get('seg_type')
    out['segments'] = segments
    return out


def _key(row):
    return (round(float(row.get('frequency_ghz', 0.0)), 9), round(float(row.get('theta_inc_deg', 0.0)), 9),
            round(float(row.get('theta_scat_deg', 0.0)), 9))


def _exact(row):
    return (float(row.get('frequency_ghz', 0.0)), float(row.get('theta_inc_deg', 0.0)),
            float(row.get('theta_scat_deg', 0.0)))


def _finite(row, key):
    if key not in row:
        raise ValueError(f'Mesh convergence requires authoritative complex amplitudes; sample {_key(row)} is missing '
                         f'{key!r}.')
    value = float(row[key])
    if not math.isfinite(value):
        raise ValueError(f'Mesh convergence sample {_key(row)} has non-finite {key}={row[key]!r}.')
    return value


def _db(row):
    if 'rcs_db' in row:
        value = float(row['rcs_db'])
    else:
        value = 10.0 * math.log10(max(_finite(row, 'rcs_linear'), EPS))
    if not math.isfinite(value):
        raise ValueError(f'Mesh convergence sample {_key(row)} has non-finite rcs_db={value!r}.')
    return value


def _matched(base_samples, fine_samples):
    """Sample pairs on the same (frequency, incidence, scattering) grid point, sorted by the
    rounded coordinates and then the exact ones."""
    def grouped(samples, label):
        out, seen = {}, set()
        for row in samples:
            ex = _exact(row)
            if ex in seen:
                raise ValueError(f'Mesh convergence {label} contains duplicate exact sample coordinates {ex}.')
            seen.add(ex)
            out.setdefault(_key(row), []).append(row)
        for rows in out.values():
            rows.sort(key=_exact)
        return out
    b, f = grouped(base_samples, 'base_result'), grouped(fine_samples, 'fine_result')
    keys = set(b) | set(f)
    missing = sum(max(0, len(b.get(k, ())) - len(f.get(k, ()))) for k in keys)
    extra = sum(max(0, len(f.get(k, ())) - len(b.get(k, ()))) for k in keys)
    if missing or extra:
        raise ValueError(f'Mesh convergence sample grids differ: {missing} missing and {extra} extra fine-result '
                         'sample point(s).')
    pairs = []
    for key in sorted(b):
        pairs.extend(zip(b[key], f[key]))
    if not pairs:
        raise ValueError('Mesh convergence comparison produced no overlapping samples.')
    return pairs


def evaluate_mesh_convergence(base_result, fine_result, rms_limit_db, max_abs_limit_db, complex_rms_limit=0.02,
                              complex_max_limit=0.05, phase_rms_limit_deg=5.0, phase_max_limit_deg=15.0,
                              phase_floor_relative=LEVEL_FLOOR, db_floor_relative=LEVEL_FLOOR):
    """Point-by-point comparison of two results' samples (runs/quality.py:265-547); returns
    the same report dict (``passed``, metrics, ``limits``, ``violations``, ``reason``)."""
    policy = validate_policy({'rms_limit_db': rms_limit_db, 'max_abs_limit_db': max_abs_limit_db,
                              'complex_rms_limit': complex_rms_limit, 'complex_max_limit': complex_max_limit,
                              'phase_rms_limit_deg': phase_rms_limit_deg, 'phase_max_limit_deg': phase_max_limit_deg,
                              'phase_floor_relative': phase_floor_relative, 'db_floor_relative': db_floor_relative})
    base_samples = base_result.get('samples', []) or []
    fine_samples = fine_result.get('samples', []) or []
    if not base_samples or not fine_samples:
        raise ValueError('Both base_result and fine_result must contain samples.')
    pairs = _matched(base_samples, fine_samples)
    base_amp = np.array([complex(_finite(r, 'rcs_amp_real'), _finite(r, 'rcs_amp_imag')) for r, _o in pairs])
    fine_amp = np.array([complex(_finite(o, 'rcs_amp_real'), _finite(o, 'rcs_amp_imag')) for _r, o in pairs])
    unfloored = np.array([_db(r) - _db(o) for r, o in pairs], dtype=float)
    groups = {}
    for i, (row, _o) in enumerate(pairs):
        groups.setdefault(round(float(row.get('frequency_ghz', 0.0)), 9), []).append(i)
    n = len(pairs)
    cerr, deltas = np.zeros(n), np.zeros(n)
    above = np.zeros(n, dtype=bool)
    phase_groups, peaks = [], {}
    dbf, phf = policy['db_floor_relative'], policy['phase_floor_relative']
    for freq, raw in sorted(groups.items()):
        idx = np.asarray(raw, dtype=int)
        ba, fa = np.abs(base_amp[idx]), np.abs(fine_amp[idx])
        peak = float(max(np.max(ba), np.max(fa)))
        peaks[str(freq)] = peak
        if not math.isfinite(peak) or peak <= 0.0:
            continue
        cerr[idx] = np.abs(base_amp[idx] - fine_amp[idx]) / peak
        floor = max(dbf * peak, np.finfo(float).tiny)
        deltas[idx] = 20.0 * (np.log10(ba + floor) - np.log10(fa + floor))
        above[idx] = np.maximum(ba, fa) >= dbf * peak
        mask = (ba > phf * peak) & (fa > phf * peak)
        if np.any(mask):
            phase_groups.append(np.abs(np.degrees(np.angle(fine_amp[idx][mask] * np.conj(base_amp[idx][mask])))))
    phase = np.concatenate(phase_groups) if phase_groups else np.zeros(0)
    absd = np.abs(deltas)
    rms_db, max_db = float(np.sqrt(np.mean(deltas * deltas))), float(np.max(absd))
    c_rms, c_max = float(np.sqrt(np.mean(cerr ** 2))), float(np.max(cerr))
    p_rms = float(np.sqrt(np.mean(phase ** 2))) if phase.size else 0.0
    p_max = float(np.max(phase)) if phase.size else 0.0
    violations = []
    checks = ((rms_db, rms_limit_db, 'RMS dB delta {v:.6g} exceeds limit {l:.6g}'),
              (max_db, max_abs_limit_db, 'Max |dB| delta {v:.6g} exceeds limit {l:.6g}'),
              (c_rms, complex_rms_limit, 'RMS normalized complex-field delta {v:.6g} exceeds limit {l:.6g}'),
              (c_max, complex_max_limit, 'Max normalized complex-field delta {v:.6g} exceeds limit {l:.6g}'),
              (p_rms, phase_rms_limit_deg, 'RMS phase delta {v:.6g} deg exceeds limit {l:.6g} deg'),
              (p_max, phase_max_limit_deg, 'Max phase delta {v:.6g} deg exceeds limit {l:.6g} deg'))
    for value, limit, text in checks:
        if value > float(limit):
            violations.append(text.format(v=value, l=float(limit)))
    return {
        'passed': not violations,
        'sample_count': int(n),
        'rms_db': rms_db,
        'max_abs_db': max_db,
        'mean_db': float(np.mean(deltas)),
        'median_abs_db': float(np.median(absd)),
        'db_metric': '20*log10(|A| + db_floor_relative*peak) per frequency',
        'db_sample_count_above_floor': int(np.count_nonzero(above)),
        'rms_db_unfloored': float(np.sqrt(np.mean(unfloored ** 2))),
        'max_abs_db_unfloored': float(np.max(np.abs(unfloored))),
        'complex_rms_normalized': c_rms,
        'complex_max_normalized': c_max,
        'complex_reference_peak_amplitude': float(max(peaks.values())),
        'complex_reference_peak_amplitude_by_frequency': peaks,
        'phase_sample_count': int(phase.size),
        'phase_rms_deg': p_rms,
        'phase_max_deg': p_max,
        'limits': {'rms_db': float(rms_limit_db), 'max_abs_db': float(max_abs_limit_db),
                   'complex_rms_normalized': float(complex_rms_limit),
                   'complex_max_normalized': float(complex_max_limit),
                   'phase_rms_deg': float(phase_rms_limit_deg), 'phase_max_deg': float(phase_max_limit_deg),
                   'phase_floor_relative': float(phf), 'db_floor_relative': float(dbf)},
        'violations': violations,
        'reason': '; '.join(violations) if violations else 'mesh convergence passed',
    }


def certify(base_result, fine_result, policy, base_panels, fine_panels):
    """Publish the refined result with its certificate (twod/solver.py ``_certify_2d_results``):
    the refined mesh must have more panels and agree with the base mesh within the policy,
    else ValueError('Certified 2-D mesh convergence failed: ...')."""
    if base_panels > 0 and fine_panels <= base_panels:
        raise ValueError(f'Certified 2-D mesh refinement failed: the fine solve used {fine_panels} panels versus '
                         f'{base_panels} on the base mesh. A mesh-convergence certificate requires a genuinely '
                         'refined discretization.')
    gate = evaluate_mesh_convergence(base_result, fine_result, policy['rms_limit_db'], policy['max_abs_limit_db'],
                                     policy['complex_rms_limit'], policy['complex_max_limit'],
                                     policy['phase_rms_limit_deg'], policy['phase_max_limit_deg'],
                                     policy['phase_floor_relative'], policy['db_floor_relative'])
    gate.update({'schema': 'ghost.solver.mesh-convergence.v1', 'fine_factor': policy['fine_factor'],
                 'published_mesh': 'fine', 'geometry_model': 'piecewise_linear_input',
                 'geometry_approximation_certified': False,
                 'base_quality_gate': dict(base_result.get('metadata', {}).get('quality_gate', {}) or {}),
                 'fine_quality_gate': dict(fine_result.get('metadata', {}).get('quality_gate', {}) or {}),
                 'refinement_kind': 'mesh', 'base_panel_count': int(base_panels),
                 'fine_panel_count': int(fine_panels),
                 'panel_refinement_ratio': float(fine_panels) / float(base_panels) if base_panels > 0 else
                 float('nan')})
    if not gate['passed']:
        raise ValueError('Certified 2-D mesh convergence failed: ' + str(gate['reason']))
    result = dict(fine_result)
    meta = dict(result.get('metadata', {}))
    meta.update(mesh_convergence=gate, mesh_convergence_certified=True, certified_entry_point=True,
                published_mesh='fine')
    qg = meta.get('quality_gate')
    if isinstance(qg, dict):
        qg = dict(qg)
        qg['mesh_convergence_certified'] = True
        qg['certification_scope'] = 'discrete_linear_system_and_mesh_convergence'
        meta['quality_gate'] = qg
    result['metadata'] = meta
    return result
