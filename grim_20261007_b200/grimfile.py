"""``.grim`` archives of monostatic solver results (the output format of the reference's
``io/grim.py:1034`` ``export_result_to_grim``; reader ``:1183`` ``load_grim_npz``).

A ``.grim`` file is a compressed NumPy archive holding one rectangular grid of the
scattered field over (azimuth, elevation, frequency, polarisation) and its metadata, the
format GRIM reads.  Format version 2 (the default; ``GHOST_GRIM_FORMAT_VERSION`` or
``format_version`` selects 1) stores each sample's complex amplitude once as
``rcs_complex`` (complex128) with the framing keys ``grim_format_version``,
``storage_kind`` and ``storage_domain``; version 1 stores float32 linear power and phase
and the float64 real and imaginary amplitude.  The metadata keys (axes, polarisation
labels, units, phase reference, amplitude convention, the solver-metadata JSON envelope)
are the reference's, so GRIM and the reference's own reader open these files.

This module restates the reference's export of the results this package's public solves
return (``twod/solver.py`` single-polarisation and co-polarised VV/HH results):
grid placement from the samples (first sample of a repeated coordinate kept, repeats
checked against it), the completeness check, the power / amplitude consistency check of
every sample, the deterministic JSON envelope (``ghost.solver_metadata.v1``) and the
atomic write.  Bistatic results (one file per incidence angle) are not produced by this
package's solves and are refused.  ``tests/golden/make_grim_golden.py`` records the
reference's own files for fixed result dicts; the tests require every stored array and
string to be equal.
"""
from __future__ import annotations

import json
import math
import os
import tempfile
from io import StringIO

import numpy as np

C0 = 299_792_458.0
EPS = 1e-12
SOLVER_METADATA_SCHEMA = 'ghost.solver_metadata.v1'
FORMAT_VERSION_ENV = 'GHOST_GRIM_FORMAT_VERSION'
_VALUE_FIELDS = ('theta_scat_deg', 'frequency_ghz', 'rcs_linear', 'rcs_amp_real', 'rcs_amp_imag')
_DIAGNOSTIC_KEYS = ('linear_residual', 'linear_backward_error', 'constraint_residual', 'constraint_residual_norm',
                    'condition_est')


def format_version(requested=None):
    """The archive layout to write: 1 or 2 (``None``: the environment setting, else 2)."""
    if requested is None:
        setting = os.environ.get(FORMAT_VERSION_ENV, '').strip()
        return int(setting) if setting in ('1', '2') else 2
    if isinstance(requested, bool) or requested not in (1, 2):
        raise ValueError(f'GRIM format_version must be 1 or 2; got {requested!r}.')
    return int(requested)


# ------------------------------------------------------------------ labels
def canonical_polarization(label):
    text = str(label or '').strip().upper()
    if text in {'TM', 'HH', 'H', 'HORIZONTAL'} or not text:
        return 'TM'
    if text in {'TE', 'VV', 'V', 'VERTICAL'}:
        return 'TE'
    raise ValueError(f"Unsupported polarization '{label}'. Use TM/HH/H/HORIZONTAL or TE/VV/V/VERTICAL.")


def _primary_alias(label):
    return 'HH' if canonical_polarization(label) == 'TM' else 'VV'


def _aliases(label):
    return ['TM', 'HH', 'H', 'HORIZONTAL'] if canonical_polarization(label) == 'TM' else ['TE', 'VV', 'V', 'VERTICAL']


# ------------------------------------------------------------------ solver-metadata envelope
def json_safe(value):
    """Deterministic, standards-compliant JSON data: non-finite floats and complex numbers
    as tagged objects, dict keys sorted, sets sorted by their JSON text."""
    if value is None or isinstance(value, (str, bool)):
        return value
    if isinstance(value, np.generic):
        return json_safe(value.item())
    if isinstance(value, int):
        return int(value)
    if isinstance(value, float):
        if math.isfinite(value):
            return float(value)
        return {'__nonfinite_float__': 'nan' if math.isnan(value) else ('infinity' if value > 0 else '-infinity')}
    if isinstance(value, complex):
        return {'__complex__': {'real': json_safe(float(value.real)), 'imag': json_safe(float(value.imag))}}
    if isinstance(value, np.ndarray):
        return json_safe(value.tolist())
    if isinstance(value, dict):
        return {str(k): json_safe(v) for k, v in sorted(value.items(), key=lambda kv: str(kv[0]))}
    if isinstance(value, (list, tuple)):
        return [json_safe(v) for v in value]
    if isinstance(value, (set, frozenset)):
        items = [json_safe(v) for v in value]
        return sorted(items, key=lambda v: json.dumps(v, sort_keys=True, separators=(',', ':'), ensure_ascii=False))
    if isinstance(value, os.PathLike):
        return os.fspath(value)
    return str(value)


def solver_metadata_json(result):
    """The audit envelope stored with every export: the result's identifying keys and
    metadata, and the per-sample diagnostics in (frequency, incidence, scattering) order."""
    samples = list(result.get('samples', []) or [])
    rows = sorted((r for r in samples if any(k in r for k in _DIAGNOSTIC_KEYS)),
                  key=lambda r: tuple(float(r.get(k)) for k in ('frequency_ghz', 'theta_inc_deg', 'theta_scat_deg')))
    envelope = {
        'schema': SOLVER_METADATA_SCHEMA,
        'solver': result.get('solver', ''),
        'scattering_mode': result.get('scattering_mode', ''),
        'polarization': result.get('polarization', ''),
        'polarization_export': result.get('polarization_export', ''),
        'polarizations': result.get('polarizations', []) or [],
        'polarization_mapping': result.get('polarization_mapping', {}) or {},
        'rcs_log_unit': result.get('rcs_log_unit', ''),
        'rcs_linear_quantity': result.get('rcs_linear_quantity', ''),
        'amplitude_convention': result.get('amplitude_convention', ''),
        'amplitude_version': result.get('amplitude_version', 1),
        'metadata': result.get('metadata', {}) or {},
        'sample_diagnostics': None,
    }
    enc = json.JSONEncoder(sort_keys=True, separators=(',', ':'), ensure_ascii=False, allow_nan=False)
    out = StringIO()
    out.write('{')
    for i, key in enumerate(sorted(envelope)):
        if i:
            out.write(',')
        out.write(enc.encode(key) + ':')
        if key != 'sample_diagnostics':
            out.write(enc.encode(json_safe(envelope[key])))
            continue
        out.write('[')
        for j, r in enumerate(rows):
            if j:
                out.write(',')
            out.write(enc.encode(json_safe(dict(frequency_ghz=r.get('frequency_ghz'),
                                                theta_inc_deg=r.get('theta_inc_deg'),
                                                theta_scat_deg=r.get('theta_scat_deg'),
                                                polarization=r.get('polarization', ''),
                                                **{k: r[k] for k in _DIAGNOSTIC_KEYS if k in r}))))
        out.write(']')
    out.write('}')
    return out.getvalue()


# ------------------------------------------------------------------ grids
def _required(row, key):
    if key not in row:
        raise ValueError(f"Solver sample is missing required field '{key}'.")
    try:
        value = float(row[key])
    except (TypeError, ValueError, OverflowError) as exc:
        raise ValueError(f"Solver sample field '{key}' must be a finite numeric value; got {row[key]!r}.") from exc
    if not math.isfinite(value):
        raise ValueError(f"Solver sample field '{key}' must be finite; got {row[key]!r}.")
    return value


def _expected_linear(quantity, freq_ghz, amp_abs2):
    if quantity == 'sigma_2d':
        return amp_abs2 / (4.0 * (2.0 * math.pi * freq_ghz * 1.0e9 / C0))
    return 4.0 * math.pi * amp_abs2


def _check_rows(samples, quantity):
    """Row-by-row validation: the first invalid sample with its message."""
    for i, row in enumerate(samples):
        try:
            vals = [_required(row, k) for k in _VALUE_FIELDS]
        except ValueError as exc:
            raise ValueError(f'Invalid solver sample at index {i}: {exc}') from exc
        _az, freq, lin, re, im = vals
        if freq <= 0.0:
            raise ValueError(f'Invalid solver sample at index {i}: frequency_ghz must be positive; got {freq!r}.')
        if lin < 0.0:
            raise ValueError(f'Invalid solver sample at index {i}: rcs_linear must be non-negative; got {lin!r}.')
        with np.errstate(over='ignore', invalid='ignore'):
            a2 = re * re + im * im
        if not math.isfinite(a2):
            raise ValueError(f'Invalid solver sample at index {i}: the finite complex amplitude is too large to '
                             'form finite physical power.')
        exp = _expected_linear(quantity, freq, a2)
        if not math.isfinite(exp):
            raise ValueError(f'Invalid solver sample at index {i}: normalized linear RCS is not finite.')
        if abs(lin - exp) > 2.0e-8 * max(exp, lin) + np.finfo(float).tiny:
            raise ValueError(f'Invalid solver sample at index {i}: rcs_linear {lin:.12g} is inconsistent with the '
                             f'complex amplitude under {quantity} normalization (expected {exp:.12g}).')


def _columns(samples, quantity):
    """The five exported values as float64 columns, every sample validated (vectorised;
    the row loop reports the first invalid one)."""
    n = len(samples)
    try:
        cols = [np.fromiter((float(r[k]) for r in samples), dtype=np.float64, count=n) for k in _VALUE_FIELDS]
    except (KeyError, TypeError, ValueError, OverflowError):
        cols = None
    if cols is not None:
        theta, freq, lin, re, im = cols
        with np.errstate(over='ignore', invalid='ignore', divide='ignore'):
            a2 = re * re + im * im
            exp = (a2 / (4.0 * (2.0 * math.pi * freq * 1.0e9 / C0)) if quantity == 'sigma_2d'
                   else 4.0 * math.pi * a2)
            bad = ~np.isfinite(theta)
            for c in (freq, lin, re, im):
                bad |= ~np.isfinite(c)
            bad |= (freq <= 0.0) | (lin < 0.0) | ~np.isfinite(a2) | ~np.isfinite(exp)
            bad |= np.abs(lin - exp) > 2.0e-8 * np.maximum(exp, lin) + np.finfo(float).tiny
        if not np.any(bad):
            return cols
    _check_rows(samples, quantity)
    raise ValueError('Invalid solver samples.')


def _channel_grid(samples, polarization, quantity, preserve_raw):
    """One polarisation's rectangular grid: axes, float32 power, phase and (raw) the
    complex field, from the first sample at each coordinate."""
    if not samples:
        raise ValueError('No samples available to export.')
    theta, freq, lin, re, im = _columns(samples, quantity)
    az = np.unique(theta)
    fr = np.unique(freq)
    shape = (len(az), 1, len(fr), 1)
    cells = np.searchsorted(az, theta) * len(fr) + np.searchsorted(fr, freq)
    uniq, first = np.unique(cells, return_index=True)
    with np.errstate(invalid='ignore'):
        phase = np.arctan2(im, re)
    phase[(re == 0.0) & (im == 0.0)] = 0.0
    dup = np.ones(cells.size, dtype=bool)
    dup[first] = False
    if np.any(dup):
        rep = np.flatnonzero(dup)
        org = first[np.searchsorted(uniq, cells[rep])]
        p_conf = np.abs(lin[org].astype(np.float32).astype(np.float64) - lin[rep]) > EPS
        ph0 = phase[org].astype(np.float32).astype(np.float64)
        d = np.remainder(phase[rep] - ph0 + math.pi, 2.0 * math.pi) - math.pi
        ph_conf = np.abs(d) > 1e-5
        conf = np.flatnonzero(p_conf | ph_conf)
        if conf.size:
            row = rep[conf[0]]
            kind = 'sample' if p_conf[conf[0]] else 'amplitude'
            raise ValueError(f'Duplicate {kind} conflict at az={theta[row]}, el=0, f={freq[row]}, pol={polarization}.')
    power = np.full(shape, np.nan, dtype=np.float32)
    power.flat[uniq] = lin[first]
    missing = np.argwhere(~np.isfinite(power))
    if missing.size:
        raise ValueError('Solver samples do not form a complete rectangular (angle x frequency x polarization) '
                         f'grid: {len(missing)} cell(s) are missing; first missing index is '
                         f'{tuple(int(v) for v in missing[0])}.')
    out = {'azimuths': az, 'frequencies': fr, 'power': power}
    if preserve_raw:
        field = np.full(shape, complex(np.nan, np.nan), dtype=np.complex128)
        field.real.flat[uniq] = re[first]
        field.imag.flat[uniq] = im[first]
        out['field'] = field
    else:
        ph = np.full(shape, np.nan, dtype=np.float32)
        ph.flat[uniq] = phase[first]
        out['phase'] = ph
    return out


def _common_metadata(quantity, log_unit, source_path, history, preserve_raw):
    units = {'azimuth': 'deg', 'elevation': 'deg', 'frequency': 'GHz', 'rcs_log_unit': str(log_unit),
             'rcs_linear_quantity': str(quantity)}
    if quantity == 'sigma_2d':
        phase_reference = ('origin=(0,0), convention=exp(+jwt); stored complex field is the 2D layer-potential '
                           'bare-integral amplitude B. The coefficient in u_s~exp(-j(kr-pi/4))/sqrt(8*pi*k*r)*A is '
                           'A=j*B.')
        domain = '2d_layer_potential_bare_integral_amplitude_B'
        convention = 'A_physical_asymptotic = +j * B_stored'
    else:
        phase_reference = 'origin=(0,0), convention=exp(+jwt), monostatic far-field amplitude'
        domain = 'solver_raw_far_field_amplitude'
        convention = 'solver physical far-field amplitude'
    meta = {'rcs_domain': 'power_phase', 'power_domain': 'linear_rcs', 'source_path': source_path,
            'history': history, 'units': json.dumps(units), 'phase_reference': phase_reference,
            'amplitude_convention': convention, 'raw_complex_amplitude_preserved': bool(preserve_raw)}
    if preserve_raw:
        meta['complex_field_domain'] = domain
    return meta


def build_payload(result, source_path='', history='', preserve_raw_complex_amplitude=True):
    """The archive content of a monostatic result: one channel, or the VV/HH pair of a
    co-polarised result (one file, polarisation axis [VV, HH])."""
    samples = result.get('samples', []) or []
    if not samples:
        raise ValueError('No solver samples were returned, nothing to export.')
    declared = [str(v).strip().upper() for v in list(result.get('polarizations', []) or [])]
    co = result.get('co_solved_samples', {}) or {}
    dual = declared == ['VV', 'HH'] and isinstance(co, dict) and set(co) == {'VV', 'HH'}
    mapping = result.get('polarization_mapping', {}) or {}
    if (declared or co) and not dual:
        raise ValueError('A declared co-polarized result must contain ordered polarizations [VV, HH] and exactly '
                         'matching co_solved_samples; single-channel fallback was refused.')
    if dual and set(mapping) != {'VV', 'HH'}:
        raise ValueError('A co-polarized result must declare its VV/HH physical mapping.')
    if str(result.get('scattering_mode', 'monostatic')).strip().lower() == 'bistatic':
        raise NotImplementedError('Bistatic results are not produced by this package and are not exported.')
    quantity = str(result.get('rcs_linear_quantity', 'sigma_2d')).strip().lower()
    if quantity not in {'sigma_2d', 'sigma_3d'}:
        raise ValueError("rcs_linear_quantity must be 'sigma_2d' or 'sigma_3d'.")
    log_unit = str(result.get('rcs_log_unit', 'dBke'))
    raw = bool(preserve_raw_complex_amplitude)
    if dual:
        chans = [_channel_grid(co[p] or [], p, quantity, raw) for p in ('VV', 'HH')]
        for name in ('azimuths', 'frequencies'):
            if not np.array_equal(chans[0][name], chans[1][name]):
                raise ValueError(f'VV and HH cannot share one GRIM file because their {name} axes differ.')
        labels = [str(mapping[c]).strip().upper() for c in ('VV', 'HH')]
        if any(not lab for lab in labels):
            raise ValueError('Co-polarized GRIM mapping labels cannot be empty.')
        pols = np.asarray(['VV', 'HH'], dtype=str)
        primary, aliases = ','.join(labels), json.dumps(labels)
        grid = {'azimuths': chans[0]['azimuths'], 'frequencies': chans[0]['frequencies'],
                'power': np.concatenate([c['power'] for c in chans], axis=-1)}
        key = 'field' if raw else 'phase'
        grid[key] = np.concatenate([c[key] for c in chans], axis=-1)
    else:
        label = canonical_polarization(result.get('polarization_export') or result.get('polarization') or 'TM')
        grid = _channel_grid(samples, label, quantity, raw)
        pols = np.asarray([_primary_alias(label)], dtype=str)
        primary, aliases = label, json.dumps(_aliases(label))
    payload = {'azimuths': grid['azimuths'], 'elevations': np.asarray([0.0], dtype=float),
               'frequencies': grid['frequencies'], 'polarizations': pols, 'polarization_alias_primary': primary,
               'polarization_aliases_json': aliases, 'power': grid['power']}
    if raw:
        payload['field'] = grid['field']
        if not np.all(np.isfinite(grid['field'].real)) or not np.all(np.isfinite(grid['field'].imag)):
            raise ValueError('Solver complex amplitudes are not finite after grid construction.')
    else:
        payload['phase'] = grid['phase']
    payload.update(_common_metadata(quantity, log_unit, source_path, history, raw))
    payload['solver_metadata_json'] = solver_metadata_json(result)
    return payload


def _power_scale2(payload):
    units = json.loads(payload['units'])
    if units.get('rcs_linear_quantity') == 'sigma_2d':
        k = 2.0 * math.pi * np.asarray(payload['frequencies'], dtype=float) * 1.0e9 / C0
        return (1.0 / (4.0 * k))[None, None, :, None]
    return 4.0 * math.pi


def _derived(payload):
    """float32 power and phase and float64 real / imaginary parts of the stored field."""
    f = payload['field']
    power = ((f.real * f.real + f.imag * f.imag) * _power_scale2(payload)).astype(np.float32)
    phase = np.where((f.real == 0.0) & (f.imag == 0.0), 0.0, np.angle(f)).astype(np.float32)
    return power, phase, np.array(f.real, dtype=np.float64), np.array(f.imag, dtype=np.float64)


def validate_payload(payload):
    """Malformed or non-finite grids are refused before the destination is opened."""
    for key in ('azimuths', 'elevations', 'frequencies'):
        axis = np.asarray(payload[key], dtype=float)
        if axis.ndim != 1 or axis.size == 0:
            raise ValueError(f"GRIM axis '{key}' must be a non-empty 1-D array.")
        if not np.all(np.isfinite(axis)):
            raise ValueError(f"GRIM axis '{key}' contains NaN or infinite values.")
        if np.any(np.diff(axis) <= 0.0):
            raise ValueError(f"GRIM axis '{key}' must be strictly increasing.")
    if np.any(np.asarray(payload['frequencies']) <= 0.0):
        raise ValueError('GRIM frequencies must be positive.')
    pols = np.asarray(payload['polarizations']).astype(str)
    if pols.ndim != 1 or pols.size == 0 or any(not p.strip() for p in pols) or len(set(pols.tolist())) != pols.size:
        raise ValueError('GRIM polarization labels must be a non-empty 1-D array of unique, non-empty labels.')
    power = payload['power']
    if not np.all(np.isfinite(power)) or np.any(power < 0):
        raise ValueError("GRIM grid 'rcs_power' contains NaN, infinite or negative values.")
    if 'field' in payload:
        dpow, dphase, _re, _im = _derived(payload)
        f = payload['field']
        live = (np.abs(f.real) > np.finfo(np.float32).tiny) | (np.abs(f.imag) > np.finfo(np.float32).tiny)
        if np.any(live):
            err = np.abs(np.angle(np.exp(1j * (dphase.astype(float)[live] - np.angle(f[live])))))
            if float(np.max(err)) > 2.0e-5:
                raise ValueError('GRIM rcs_phase is inconsistent with its stored complex amplitude.')
        a2 = f.real * f.real + f.imag * f.imag
        expected = a2 * _power_scale2(payload)
        tol = 16.0 * np.finfo(np.float32).eps * np.maximum(expected, power) + np.finfo(np.float32).tiny
        if np.any(np.abs(power.astype(float) - expected) > tol):
            raise ValueError('GRIM rcs_power is inconsistent with its stored complex amplitude.')


def save_payload(payload, path, version=None):
    """Write ``payload`` atomically as ``path`` (``.grim`` appended when missing); returns
    the path written.  Version 2 with a stored field: ``rcs_complex`` only; otherwise the
    version-1 arrays."""
    version = format_version(version)
    validate_payload(payload)
    out = path if path.lower().endswith('.grim') else f'{path}.grim'
    folder = os.path.dirname(os.path.abspath(out))
    os.makedirs(folder, exist_ok=True)
    fd, tmp = tempfile.mkstemp(prefix=f'.{os.path.basename(out)}.', suffix='.tmp', dir=folder)
    os.close(fd)
    raw = 'field' in payload
    arrays = {k: payload[k] for k in ('azimuths', 'elevations', 'frequencies', 'polarizations',
                                      'polarization_alias_primary', 'polarization_aliases_json')}
    if not (version == 2 and raw):
        if raw:
            _dp, phase, _re, _im = _derived(payload)
        else:
            phase = payload['phase']
        arrays['rcs_power'] = payload['power']
        arrays['rcs_phase'] = phase
    for k in ('rcs_domain', 'power_domain', 'source_path', 'history', 'units', 'phase_reference',
              'amplitude_convention', 'raw_complex_amplitude_preserved'):
        arrays[k] = payload[k]
    if raw:
        if version == 2:
            arrays.update(grim_format_version=np.int16(2), storage_kind='complex', storage_domain='raw_field',
                          rcs_complex=payload['field'])
        else:
            _dp, _ph, re, im = _derived(payload)
            arrays['rcs_amp_real'], arrays['rcs_amp_imag'] = re, im
        arrays['complex_field_domain'] = payload['complex_field_domain']
    arrays['solver_metadata_json'] = payload['solver_metadata_json']
    try:
        with open(tmp, 'wb') as fh:
            np.savez_compressed(fh, **arrays)
            fh.flush()
            os.fsync(fh.fileno())
        os.replace(tmp, out)
    except BaseException:
        try:
            os.unlink(tmp)
        except FileNotFoundError:
            pass
        raise
    return out


def export_result_to_grim(result, output_path, source_path='', history='', preserve_raw_complex_amplitude=True,
                          format_version=None):
    """Export a monostatic solver result (single polarisation, or the VV/HH pair of a
    co-polarised solve) as one ``.grim`` archive; returns ``[absolute path]``
    (the reference's signature and return)."""
    payload = build_payload(result, source_path, history, preserve_raw_complex_amplitude)
    return [os.path.abspath(save_payload(payload, output_path, format_version))]


def load_grim_npz(path):
    """Read a ``.grim`` archive as the version-1 key set: a version-2 ``rcs_complex``
    archive gives float32 ``rcs_power`` / ``rcs_phase`` and float64 ``rcs_amp_real`` /
    ``rcs_amp_imag`` derived from the field; the framing keys are dropped."""
    with np.load(path, allow_pickle=False) as data:
        arrays = {k: data[k] for k in data.files}
    if 'grim_format_version' not in arrays:
        return arrays
    version = int(np.asarray(arrays.pop('grim_format_version')).reshape(-1)[0])
    if version == 1:
        return arrays
    kind = str(np.asarray(arrays.pop('storage_kind')).reshape(-1)[0])
    domain = str(np.asarray(arrays.pop('storage_domain')).reshape(-1)[0])
    if kind != 'complex' or domain != 'raw_field':
        raise ValueError(f'{path}: storage {kind!r}/{domain!r} is not written by this package.')
    payload = {'field': arrays.pop('rcs_complex'), 'units': str(arrays['units']), 'frequencies': arrays['frequencies']}
    arrays['rcs_power'], arrays['rcs_phase'], arrays['rcs_amp_real'], arrays['rcs_amp_imag'] = _derived(payload)
    return arrays
