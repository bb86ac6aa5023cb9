"""2-D monostatic RCS on the GPU, behind the reference's solver entry points.

Public API (same names, arguments and result-dict keys as the reference):

* ``solve_monostatic_rcs_2d(geometry_snapshot, frequencies_ghz, elevations_deg, ...)``
  -- ``twod/solver.py:3193``: both co-polarised channels (VV = TE, HH = TM), samples
  interleaved VV then HH per physical sample, ``co_solved_samples`` per channel
  (``_merge_co_polarized_2d_results`` ``:2778``);
* ``solve_monostatic_rcs_2d_single_polarization(...)`` -- ``twod/solver.py:1988``;
* ``_solve_dense_gpu(a_eval, rhs_eval) -> (x, device_name)`` -- ``twod/solver.py:355``,
  the ``GHOST_DENSE_BACKEND=gpu`` hook (CuPy cuSOLVER there, libgrimgpu here);
* ``_solve_dense_system(a_mat, rhs, ...)`` -- ``twod/solver.py:613-773``: GPU solve,
  then the FP64 normwise backward-error gate (1e-12) with at most two refinement
  steps, raising ``RuntimeError`` when the gate fails.

Physics: the reference's own discretisation of closed PEC contours (``galerkin.py``):
linear Galerkin elements, combined rows S + gamma (D + M/2) (TM) and K' - M/2 - gamma W
(TE), so the amplitudes equal the reference solver's to rounding and conditioning
(1e-10 on its C1 cylinder) and neither channel has interior resonances.  The
pulse-basis, point-matched TM EFIE / TE MFIE of ``operators.DeviceBody`` remains
selectable with ``GRIM_2D_FORMULATION=pulse`` (it agrees with the reference only to
discretisation error).
"""
from __future__ import annotations

import concurrent.futures as cf
import math
import os
import threading
import time

import numpy as np
import torch

from .. import _lib
from ..device import context, require_cuda, run_pool
from .. import sharding
from ..execution import require_gpu_dense_backend, requested_precision, requested_shard_group
from . import certify, quality
from . import galerkin
from . import geometry as geo
from . import operators as ops

C0 = 299_792_458.0
ETA0 = 376.730313668
EPS = 1e-12
RCS_NORM_NUMERATOR = 0.25
RCS_AMPLITUDE_CONVENTION = "A_physical_asymptotic = +j * B_stored"
RCS_AMPLITUDE_VERSION = 2
DENSE_LINEAR_BACKWARD_ERROR_MAX = 1.0e-12
MAX_PANELS_DEFAULT = 20_000
DEFAULT_PANELS_PER_WAVELENGTH = 20

_DENSE_BACKEND_LOCAL = threading.local()

FORMULATION_ENV = 'GRIM_2D_FORMULATION'
_FORMULATIONS = {'galerkin', 'pulse'}


def requested_formulation():
    """'galerkin' (default: the reference's linear-Galerkin combined rows) or 'pulse'."""
    value = os.environ.get(FORMULATION_ENV, 'galerkin').strip().lower()
    if value not in _FORMULATIONS:
        raise ValueError(f'{FORMULATION_ENV} must be galerkin or pulse.')
    return value


# ------------------------------------------------------------------ telemetry
def _reset_dense_backend_telemetry():
    _DENSE_BACKEND_LOCAL.events = []


def _record_dense_backend_event(**event):
    events = getattr(_DENSE_BACKEND_LOCAL, 'events', None)
    if events is None:
        events = []
        _DENSE_BACKEND_LOCAL.events = events
    events.append(dict(event))


def _dense_backend_summary():
    events = list(getattr(_DENSE_BACKEND_LOCAL, 'events', []) or [])
    used = sorted({str(e.get('used', 'gpu_grim')) for e in events})
    devices = []
    for e in events:
        d = str(e.get('gpu_device', '') or '')
        if d and d not in devices:
            devices.append(d)
    return {
        'linear_backend': used[0] if len(used) == 1 else ('mixed' if used else 'gpu_grim'),
        'dense_gpu_solve_count': sum(1 for e in events if str(e.get('used', '')).startswith('gpu')),
        'dense_cpu_solve_count': 0,
        'dense_factorization_count': sum(int(e.get('factorizations', 1)) for e in events),
        'dense_rhs_batch_count': len(events),
        'dense_rhs_column_count': sum(int(e.get('rhs_columns', 0)) for e in events),
        'dense_max_rhs_columns': max([int(e.get('rhs_columns', 0)) for e in events] or [0]),
        'dense_mixed_precision_solve_count': sum(1 for e in events if e.get('precision') == 'mixed'),
        'dense_grouped_factorization_count': sum(1 for e in events if e.get('grouped_factorization')),
        'dense_fallback_reasons': [],
        'dense_gpu_fallback_reasons': [],
        'dense_gpu_devices': devices,
        'dense_largest_system': max([int(e.get('n', 0)) for e in events] or [0]),
        'dense_pivoted_panels': sum(int(e.get('pivoted_panels', 0)) for e in events),
    }


# ------------------------------------------------------------------ dense hook (B1)
def _solve_dense_gpu(a_eval, rhs_eval):
    """GPU dense solve of A X = B for every RHS column; returns (x, device_name).

    Same contract as the reference hook: inputs are borrowed NumPy arrays
    (complex128, A n x n, B n or n x k), the solution is newly owned complex128 of
    B's shape.  Raises ``MemoryError`` when the estimated device need exceeds 80% of
    the free memory and ``RuntimeError`` on any device failure.
    """
    require_cuda()
    a = np.asarray(a_eval, dtype=np.complex128)
    b = np.asarray(rhs_eval, dtype=np.complex128)
    if a.ndim != 2 or a.shape[0] != a.shape[1]:
        raise ValueError('GPU dense solve needs a square matrix.')
    vec = b.ndim == 1
    b2 = b[:, None] if vec else b
    if b2.shape[0] != a.shape[0]:
        raise ValueError('Right-hand side height must match the matrix.')
    ctx = context()
    free, _total = ctx.mem_info()
    required = int(4.0 * a.nbytes + 3.0 * b2.nbytes + 64.0 * 1024.0 ** 2)
    if required > 0.8 * float(free):
        raise MemoryError(
            f'GPU dense solve needs an estimated {required / 1024.0 ** 3:.3f} GiB, exceeding 80% of the '
            f'{float(free) / 1024.0 ** 3:.3f} GiB currently free.')
    n, nrhs = a.shape[0], b2.shape[1]
    a_f = np.asfortranarray(a)
    x = np.array(b2, dtype=np.complex128, order='F', copy=True)
    info = _lib.ctypes.c_int(0)
    mode = _lib.PREC_MIXED if requested_precision() == 'mixed' else _lib.PREC_FP64
    try:
        torch.cuda.current_stream().synchronize()
        status = ctx.lib.grim_zgesv_batched(ctx.h, n, nrhs, a_f.ctypes.data_as(_lib.c_void_p), n,
                                            x.ctypes.data_as(_lib.c_void_p), n, mode, _lib.ctypes.byref(info))
        if status == _lib.GRIM_ERR_NOT_CONVERGED and mode == _lib.PREC_MIXED:
            # mixed -> double ladder (reference linalg/dense.py:74-98)
            x[...] = b2
            status = ctx.lib.grim_zgesv_batched(ctx.h, n, nrhs, a_f.ctypes.data_as(_lib.c_void_p), n,
                                                x.ctypes.data_as(_lib.c_void_p), n, _lib.PREC_FP64,
                                                _lib.ctypes.byref(info))
        _lib.check(status, 'grim_zgesv_batched')
    except _lib.GrimMemoryError as exc:
        raise MemoryError(str(exc)) from exc
    except _lib.GrimError as exc:
        raise RuntimeError(f'GPU dense solve failed: {exc}') from exc
    st = _lib.GrimSolveInfo()
    ctx.lib.grim_last_solve_info(ctx.h, _lib.ctypes.byref(st))
    _DENSE_BACKEND_LOCAL.last_info = st.as_dict()
    sol = x[:, 0].copy() if vec else np.ascontiguousarray(x) if b.flags.c_contiguous else x
    return np.asarray(sol, dtype=np.complex128), ctx.device_name


def matrix_inf_norm(a):
    return float(np.max(np.sum(np.abs(a), axis=1))) if a.size else 0.0


def _solve_dense_system(a_mat, rhs, condition_diagnostics=None, label='dense system', residual_diagnostics=None):
    """GPU solve + the reference's FP64 backward-error gate (``twod/solver.py:613-773``)."""
    a_eval = np.asarray(a_mat, dtype=np.complex128)
    rhs_eval = np.asarray(rhs, dtype=np.complex128)
    if not (np.all(np.isfinite(a_eval)) and np.all(np.isfinite(rhs_eval))):
        raise FloatingPointError(f'{label} contains non-finite values.')
    requested = require_gpu_dense_backend()
    solution, device = _solve_dense_gpu(a_eval, rhs_eval)
    matrix_inf = matrix_inf_norm(a_eval)

    def backward_metrics(candidate):
        x_columns = np.asarray(candidate, dtype=np.complex128)
        b_columns = rhs_eval
        if x_columns.ndim == 1:
            x_columns = x_columns[:, None]
            b_columns = b_columns[:, None]
        residual = a_eval @ x_columns - b_columns
        r = np.max(np.abs(residual), axis=0)
        den = matrix_inf * np.max(np.abs(x_columns), axis=0) + np.max(np.abs(b_columns), axis=0)
        err = np.divide(r, den, out=np.zeros_like(r), where=den > 0)
        err[(den <= 0) & (r > 0)] = math.inf
        return residual, float(np.max(err))

    residual_matrix, berr = backward_metrics(solution)
    steps = 0
    lu = None
    for _ in range(2):
        if berr <= DENSE_LINEAR_BACKWARD_ERROR_MAX:
            break
        corr_rhs = -residual_matrix if np.asarray(solution).ndim > 1 else -residual_matrix[:, 0]
        corr, _dev = _solve_dense_gpu(a_eval, corr_rhs)
        cand = solution + corr
        cand_res, cand_err = backward_metrics(cand)
        if cand_err >= berr:
            break
        solution, residual_matrix, berr, steps = cand, cand_res, cand_err, steps + 1
    if not math.isfinite(berr):
        raise RuntimeError(f'{label} produced a non-finite normwise backward error.')
    if berr > DENSE_LINEAR_BACKWARD_ERROR_MAX:
        raise RuntimeError(f'{label} normwise backward error {berr:.6g} exceeds the release limit '
                           f'{DENSE_LINEAR_BACKWARD_ERROR_MAX:.6g}.')
    info = dict(getattr(_DENSE_BACKEND_LOCAL, 'last_info', {}) or {})
    _record_dense_backend_event(requested=requested, used='gpu_grim', factorizations=1,
                                rhs_columns=1 if rhs_eval.ndim == 1 else rhs_eval.shape[1], n=a_eval.shape[0],
                                label=str(label), gpu_device=device, refinement_steps=steps,
                                precision=requested_precision(), pivoted_panels=info.get('pivoted_panels', 0))
    if condition_diagnostics is not None:
        condition_diagnostics['linear_backward_error'] = berr
        condition_diagnostics['linear_backward_error_limit'] = DENSE_LINEAR_BACKWARD_ERROR_MAX
        condition_diagnostics['linear_refinement_steps'] = steps
    if residual_diagnostics is not None:
        b_columns = rhs_eval[:, None] if rhs_eval.ndim == 1 else rhs_eval
        norm = np.linalg.norm(b_columns, axis=0)
        residual_diagnostics['relative_residual'] = np.linalg.norm(residual_matrix, axis=0) / np.where(norm <= EPS, 1., norm)
    return np.asarray(solution, dtype=np.complex128)


# ------------------------------------------------------------------ RCS helpers
def _rcs_sigma_from_amp(amp_vec, k_value):
    amp = np.asarray(amp_vec, dtype=np.complex128)
    if not np.all(np.isfinite(amp.real) & np.isfinite(amp.imag)):
        raise FloatingPointError('Far-field amplitude contains non-finite value(s).')
    k = float(k_value)
    if not math.isfinite(k) or k <= 0.0:
        raise ValueError(f'RCS normalization requires positive finite k; got {k_value!r}.')
    return np.asarray(RCS_NORM_NUMERATOR / k * np.abs(amp) ** 2, dtype=float)


def _rcs_db_from_sigma(sigma_linear, floor_linear=EPS):
    s = np.asarray(sigma_linear, dtype=float)
    if not np.all(np.isfinite(s)) or np.any(s < 0.0):
        raise ValueError('Linear RCS must contain finite non-negative values.')
    return np.asarray(10.0 * np.log10(np.maximum(s, float(floor_linear))), dtype=float)


def _canonical_user_polarization_label(label):
    text = str(label or '').strip().upper()
    if text in {'TM', 'HH', 'H', 'HORIZONTAL'}:
        return 'TM'
    if text in {'TE', 'VV', 'V', 'VERTICAL'}:
        return 'TE'
    return text


# ------------------------------------------------------------------ public solves
def _validate_request(frequencies_ghz, elevations_deg, cfie_alpha, compute_condition_number, quality_thresholds=None):
    if not frequencies_ghz:
        raise ValueError('At least one frequency is required.')
    if not elevations_deg:
        raise ValueError('At least one elevation angle is required.')
    freqs = [float(f) for f in frequencies_ghz]
    elevs = [float(e) for e in elevations_deg]
    if any((not math.isfinite(f)) or f <= 0.0 for f in freqs):
        raise ValueError('Frequencies must be positive finite GHz values.')
    if any(not math.isfinite(e) for e in elevs):
        raise ValueError('Elevation angles must all be finite.')
    if not math.isfinite(float(cfie_alpha)) or float(cfie_alpha) != 0.0:
        raise ValueError('cfie_alpha is not implemented by any active 2-D formulation; use cfie_alpha=0.')
    quality.merged_thresholds(quality_thresholds)  # unknown or invalid limits fail before any solve
    return freqs, elevs


class _MeshCache:
    """Meshes of one request, shared by the systems that use the same frequency (both
    polarisations of a co-polarised solve mesh the contour once)."""

    def __init__(self, geometry_snapshot, geometry_units, max_panels, mesh_reference_ghz, deferred_checks=False):
        self.args = (geometry_snapshot, geometry_units, max_panels, mesh_reference_ghz)
        self.lock = threading.Lock()
        self.locks = {}
        self.meshes = {}
        self.bodies = {}
        # deferred_checks: the reference's geometry checks (they depend on the snapshot only) are
        # not run while meshing; the first mesh keeps them in self.checks for the caller
        self.deferred = bool(deferred_checks)
        self.checks = []

    def galerkin_body(self, f):
        """The frequency's linear-Galerkin device body, built once and shared by both
        polarisations (its near-pair structure depends on the mesh only)."""
        polys, _geom = self.get(f)
        with self.lock:
            lk = self.locks.setdefault(('galerkin', f), threading.Lock())
        with lk:
            if f not in self.bodies:
                dev = torch.device('cuda', torch.cuda.current_device())
                body = galerkin.GalerkinBody(polys, device=dev)
                torch.cuda.current_stream().synchronize()  # other workers' streams read it next
                self.bodies[f] = body
            return self.bodies[f]

    def get(self, f):
        with self.lock:
            lk = self.locks.setdefault(f, threading.Lock())
        with lk:
            if f not in self.meshes:
                snapshot, units, max_panels, ref_ghz = self.args
                mesh_lambda = C0 / (float(ref_ghz) * 1e9) if ref_ghz else C0 / (f * 1e9)
                pending = [] if self.deferred else None
                polys = geo.contours_from_snapshot(snapshot, units, mesh_lambda, max_panels, checks=pending)
                with self.lock:
                    if pending and not self.checks:
                        self.checks.extend(pending)
                self.meshes[f] = (polys, geo.panel_geometry(polys))
            return self.meshes[f]


def _frequency_body(meshes, f, pol, abort_event):
    """(wavenumber, device body) of one (frequency, polarisation) system."""
    if abort_event is not None and abort_event.is_set():
        raise InterruptedError('Solve canceled by user.')
    k = 2.0 * math.pi * f * 1e9 / C0
    if requested_formulation() == 'galerkin':
        return k, meshes.galerkin_body(f)
    polys, geom = meshes.get(f)
    te_diag = geo.te_curvature_correction(polys) if pol == 'TE' else None
    dev = torch.device('cuda', torch.cuda.current_device())
    return k, ops.DeviceBody(geom, te_diag, device=dev)


def _frequency_record(f, elevs, pol, precision, k, body, res, t0):
    """Host samples and telemetry of one solved (frequency, polarisation) system."""
    amp = res['amplitude'].cpu().numpy()
    tele = res['telemetry']
    berr = tele.get('backward_error_dev')
    if berr is not None:
        berr_h = berr.cpu().numpy()
        if not np.all(np.isfinite(berr_h)):
            raise RuntimeError('GPU solve produced a non-finite normwise backward error.')
        if np.max(berr_h) > DENSE_LINEAR_BACKWARD_ERROR_MAX:
            raise RuntimeError(f'GPU solve normwise backward error {np.max(berr_h):.6g} exceeds the release '
                               f'limit {DENSE_LINEAR_BACKWARD_ERROR_MAX:.6g}.')
        resid = berr_h
    else:
        resid = np.full(len(elevs), float(tele.get('backward_error', 0.0)))
    sig = _rcs_sigma_from_amp(amp, k)
    sdb = _rcs_db_from_sigma(sig)
    phase = np.degrees(np.angle(amp))
    samples = [{
        'frequency_ghz': f, 'theta_inc_deg': e, 'theta_scat_deg': e,
        'rcs_linear': sl, 'rcs_db': sd, 'rcs_amp_real': ar, 'rcs_amp_imag': ai,
        'rcs_amp_phase_deg': ph, 'linear_residual': rr,
    } for e, sl, sd, ar, ai, ph, rr in zip(elevs, np.asarray(sig, dtype=float).tolist(),
                                           np.asarray(sdb, dtype=float).tolist(), amp.real.tolist(),
                                           amp.imag.tolist(), phase.tolist(), np.asarray(resid, float).tolist())]
    kind = 'galerkin' if isinstance(body, galerkin.GalerkinBody) else 'pulse'
    event = dict(requested='gpu', used='gpu_grim', factorizations=1, rhs_columns=len(elevs), n=body.n,
                 label=f'{pol} {kind} {f:g} GHz', gpu_device=context().device_name, precision=precision,
                 pivoted_panels=tele.get('pivoted_panels', 0), refinement_steps=tele.get('refinement_steps', 0),
                 grouped_factorization=bool(tele.get('grouped', False)))
    return dict(samples=samples, residuals=[float(r) for r in resid], event=event, n=body.n,
                seconds=time.perf_counter() - t0, condition_est=tele.get('condition_est'))


def _solve_frequency(meshes, f, elevs, pol, precision, abort_event, condition=False):
    """One (frequency, polarisation) system on the current device worker: mesh, fill,
    solve, far field (and, with ``condition``, the condition estimate of its FP64 matrix);
    returns host samples and telemetry."""
    t0 = time.perf_counter()
    k, body = _frequency_body(meshes, f, pol, abort_event)
    angles = np.asarray(elevs, dtype=np.float64)
    angles_dev = torch.as_tensor(angles, device=body.geom.device)
    res = ops.monostatic_solve(body, k, angles, pol, precision=precision, angles_dev=angles_dev, condition=condition)
    return _frequency_record(f, elevs, pol, precision, k, body, res, t0)


def _solve_frequencies_grouped(items, elevs, precision, abort_event, workers, condition=False):
    """Every (mesh, polarisation, frequency) system of a request through one grouped
    factorization (``operators.monostatic_solves_grouped``); returns the per-system outputs of
    ``_solve_frequency`` in ``items`` order."""
    t0 = time.perf_counter()
    keys = [(pol, f) for _m, pol, f in items]
    built = run_pool([(lambda m=m, f=f, pol=pol: _frequency_body(m, f, pol, abort_event)) for m, pol, f in items],
                     workers=workers)
    angles = np.asarray(elevs, dtype=np.float64)
    angles_dev = torch.as_tensor(angles, device=built[0][1].geom.device)
    res = ops.monostatic_solves_grouped([b for _k, b in built], [k for k, _b in built], angles,
                                        [pol for pol, _f in keys], precision=precision, angles_dev=angles_dev,
                                        workers=workers, condition=condition)
    if abort_event is not None and abort_event.is_set():
        raise InterruptedError('Solve canceled by user.')
    return [_frequency_record(f, elevs, pol, precision, k, body, r, t0)
            for (pol, f), (k, body), r in zip(keys, built, res)]


def _frequency_cost(geometry_snapshot, geometry_units, f, n_angles):
    """Relative cost of one frequency's system (N^3 + N^2 R, N from the panel density)."""
    try:
        # a cost estimate only: the geometry checks run once for the request elsewhere
        per = geo.contours_from_snapshot(geometry_snapshot, geometry_units, C0 / (f * 1e9), 10 ** 9, checks=[])
        n = sum(len(p) for p in per)
    except Exception:  # noqa: BLE001 - a costing failure only changes the order
        n = 1
    return float(n) ** 3 + float(n) ** 2 * n_angles


def _channel_result(pol, outs, precision, stage_seconds, condition=False, thresholds=None):
    """Assemble one polarisation's reference-shaped result from its per-frequency outputs,
    with the reference's quality gate (``quality.evaluate_quality_gate``) on its metadata."""
    _reset_dense_backend_telemetry()
    samples, residuals, counts, conds = [], [], [], []
    for o in outs:
        samples.extend(o['samples'])
        residuals.extend(o['residuals'])
        counts.append(o['n'])
        if o.get('condition_est') is not None:
            conds.append(float(o['condition_est']))
        _record_dense_backend_event(**o['event'])
    finite = [r for r in residuals if math.isfinite(r)]
    if requested_formulation() == 'galerkin':
        formulation = ('2D combined-field BIE, linear Galerkin (TM: S + gamma (D + M/2))' if pol == 'TM'
                       else "2D combined-field BIE, linear Galerkin (TE: K' - M/2 - gamma W)")
    else:
        formulation = 'pulse_point_matched_efie' if pol == 'TM' else 'pulse_point_matched_mfie'
    metadata = {
        'solver_method': 'direct',
        'formulation': formulation,
        'formulation_kind': 'multi_region' if requested_formulation() == 'galerkin' else 'pulse',
        'precision': precision,
        'device': context().device_name,
        'panel_count_max': max(counts),
        'panel_count_min': min(counts),
        'residual_norm_max': max(finite) if finite else float('nan'),
        'residual_norm_mean': float(np.mean(finite)) if finite else float('nan'),
        'residual_nonfinite_count': len(residuals) - len(finite),
        'constraint_residual_norm_max': 0.0,
        'junction_constraints_applied': False,
        'condition_est_max': max(conds) if conds else float('nan'),
        'condition_est_mean': float(np.mean(conds)) if conds else float('nan'),
        'condition_est_computed': bool(condition),
        'condition_estimator': 'equilibrated_1norm_lu_hager_higham' if condition else 'not_requested',
        'warnings': [],
        'runtime_profile': {'stage_seconds': stage_seconds},
        'amplitude_version': RCS_AMPLITUDE_VERSION,
        **_dense_backend_summary(),
    }
    gate = quality.evaluate_quality_gate(metadata, thresholds)
    # the solve's own backward-error gate (FP64: the reference's 1e-12; mixed: 10x its target)
    berr_limit = DENSE_LINEAR_BACKWARD_ERROR_MAX if precision == 'double' else ops.MIXED_RCS_TOL * 10
    if not (finite and max(finite) <= berr_limit):
        gate['violations'].append(f'backward error {max(finite) if finite else float("nan"):.6g} exceeds '
                                  f'{berr_limit:.6g}')
        gate['passed'] = False
        gate['reason'] = '; '.join(gate['violations'])
    metadata['quality_gate'] = gate
    return {
        'solver': '2d_bie_mom_rcs',
        'scattering_mode': 'monostatic',
        'amplitude_convention': RCS_AMPLITUDE_CONVENTION,
        'amplitude_version': RCS_AMPLITUDE_VERSION,
        'polarization': pol,
        'polarization_export': pol,
        'samples': samples,
        'metadata': metadata,
    }


def _sweep(geometry_snapshot, frequencies_ghz, elevations_deg, pols, geometry_units, progress_callback,
           cfie_alpha, compute_condition_number, max_panels, mesh_reference_ghz, abort_event, quality_thresholds=None):
    """Solve every (polarisation, frequency) system of a request on the device worker pool;
    returns {pol: reference-shaped channel result}."""
    channels = _sweep_many([geometry_snapshot], frequencies_ghz, elevations_deg, pols, geometry_units,
                           progress_callback, cfie_alpha, compute_condition_number, max_panels, mesh_reference_ghz,
                           abort_event, quality_thresholds)[0]
    for ch in channels.values():
        ch.pop('_outs', None)
    return channels


def _sweep_many(snapshots, frequencies_ghz, elevations_deg, pols, geometry_units, progress_callback, cfie_alpha,
                compute_condition_number, max_panels, mesh_reference_ghz, abort_event, quality_thresholds=None):
    """Every (snapshot, polarisation, frequency) system of a request: one grouped
    factorization of all of them when there is more than one frequency or snapshot (a
    sweep, a certified base/refined pair), else the device worker pool.  Returns, per
    snapshot, {pol: reference-shaped channel result} (with the per-system outputs under
    ``'_outs'``)."""
    freqs, elevs = _validate_request(frequencies_ghz, elevations_deg, cfie_alpha, compute_condition_number,
                                     quality_thresholds)
    condition = bool(compute_condition_number)
    require_gpu_dense_backend()
    require_cuda()
    precision = requested_precision()
    mesh_list = [_MeshCache(snap, geometry_units, max_panels, mesh_reference_ghz, deferred_checks=True)
                 for snap in snapshots]
    # each snapshot parsed and meshed here (its format errors raise now); the reference's geometry
    # checks of every snapshot then run on a host thread while the systems are solved, and
    # their error, if any, is raised before any result is returned
    for meshes in mesh_list:
        meshes.get(freqs[0])
    checks = [c for meshes in mesh_list for c in meshes.checks]
    check_pool = cf.ThreadPoolExecutor(max_workers=1) if checks else None
    check_done = check_pool.submit(lambda: [c() for c in checks]) if checks else None
    items, jobs = [], []
    for si, meshes in enumerate(mesh_list):
        for pol in pols:
            for f in freqs:
                items.append((si, pol, f))
                jobs.append(lambda m=meshes, f=f, pol=pol: _solve_frequency(m, f, elevs, pol, precision, abort_event,
                                                                           condition))
    # longest-processing-time order needs costs only when the systems differ (more than one
    # frequency or snapshot) or when they are split over ranks; each distinct (snapshot,
    # frequency) is costed once
    shard, group = requested_shard_group()
    costs = None
    if len(freqs) > 1 or len(snapshots) > 1 or shard:
        per = {}
        for si, _pol, f in items:
            if (si, f) not in per:
                per[(si, f)] = _frequency_cost(snapshots[si], geometry_units, f, len(elevs))
        costs = [per[(si, f)] for si, _pol, f in items]
    total = len(jobs) * (len(elevs) + 1)
    progress_state = {'done': 0}

    def on_done(i, out):
        progress_state['done'] += len(elevs) + 1
        if progress_callback is not None:
            _si, pol, f = items[i]
            try:
                progress_callback(progress_state['done'], total, f'{pol} solved {f:g} GHz')
            except Exception:  # noqa: BLE001 - progress reporting never fails a solve
                pass

    def run_local(idx):
        # the systems ``idx`` (indices into items) on this process's device
        idx = list(idx)
        if len(idx) > 1 and (len(freqs) > 1 or len(snapshots) > 1) and _grouped_sweeps():
            # every system through one grouped factorization (one CUDA graph)
            outs = _solve_frequencies_grouped([(mesh_list[items[i][0]], items[i][1], items[i][2]) for i in idx],
                                              elevs, precision, abort_event, sweep_workers(len(idx)), condition)
            for i, o in zip(idx, outs):
                on_done(i, o)
            return outs
        return run_pool([jobs[i] for i in idx], workers=sweep_workers(len(idx)),
                        costs=None if costs is None else [costs[i] for i in idx],
                        on_done=lambda li, o: on_done(idx[li], o))

    t0 = time.perf_counter()
    try:
        if shard:
            # this rank's LPT share of the systems, then every rank's host records
            outs = sharding.run_sharded(costs, run_local, group)
        else:
            outs = run_local(range(len(items)))
    finally:
        if check_done is not None:
            try:
                check_done.result()  # a geometry error takes precedence over anything the solve raised
            finally:
                check_pool.shutdown(wait=False)
    wall = time.perf_counter() - t0
    results = []
    for si in range(len(snapshots)):
        channels = {}
        for pol in pols:
            mine = [o for (sj, p, _f), o in zip(items, outs) if sj == si and p == pol]
            stage = {'operators': 0.0, 'linear_solve': sum(o['seconds'] for o in mine), 'far_field': 0.0,
                     'wall': wall}
            channels[pol] = _channel_result(pol, mine, precision, stage, condition, quality_thresholds)
            channels[pol]['_outs'] = mine
        results.append(channels)
    return results


def _grouped_sweeps():
    """Multi-frequency requests use the grouped factorization unless GRIM_GROUPED_SWEEP=0."""
    return os.environ.get('GRIM_GROUPED_SWEEP', '1') != '0'


def sweep_workers(njobs):
    """Device workers for a request: GRIM_SWEEP_WORKERS (default 4), at most one per system."""
    try:
        w = int(os.environ.get('GRIM_SWEEP_WORKERS', '4'))
    except ValueError:
        w = 4
    return max(1, min(w, njobs))


def solve_monostatic_rcs_2d_single_polarization(
        geometry_snapshot, frequencies_ghz, elevations_deg, polarization, geometry_units="inches",
        material_base_dir=None, progress_callback=None, quality_thresholds=None, strict_quality_gate=True,
        compute_condition_number=False, max_panels=MAX_PANELS_DEFAULT, mesh_reference_ghz=None,
        rcs_normalization_mode="physical", cfie_alpha=0.0, abort_event=None, solver_method="auto",
        _shared_discretization_cache=None):
    """Single-polarization monostatic 2-D solve on the GPU (reference ``twod/solver.py:1988``).

    Angle convention (coming-from): 0 deg arrives from the right, +90 deg from the top.
    ``linear_precision('mixed')`` selects the mixed-precision path (complex64 fill and
    LU, FP64 refinement); the default is the FP64 drop-in.  A frequency sweep runs its
    systems on a pool of device workers (``GRIM_SWEEP_WORKERS``, largest system first),
    the analogue of the reference's frequency workers (``execution/frequency_sweep.py``);
    samples are returned in frequency order.
    """
    pol = _canonical_user_polarization_label(polarization)
    if pol not in ('TM', 'TE'):
        raise ValueError(f'Unknown polarization {polarization!r}.')
    out = _sweep(geometry_snapshot, frequencies_ghz, elevations_deg, [pol], geometry_units, progress_callback,
                 cfie_alpha, compute_condition_number, max_panels, mesh_reference_ghz, abort_event,
                 quality_thresholds)[pol]
    if strict_quality_gate and not out['metadata']['quality_gate']['passed']:
        raise ValueError('Quality gate failed: ' + out['metadata']['quality_gate']['reason'])
    return out


_CO_POLARIZED_2D_CHANNELS = (('VV', 'TE'), ('HH', 'TM'))


def solve_monostatic_rcs_2d(geometry_snapshot, frequencies_ghz, elevations_deg, geometry_units="inches",
                            material_base_dir=None, progress_callback=None, quality_thresholds=None,
                            strict_quality_gate=True, compute_condition_number=False, max_panels=MAX_PANELS_DEFAULT,
                            mesh_reference_ghz=None, rcs_normalization_mode="physical", abort_event=None,
                            solver_method="auto"):
    """Both physical co-polarised channels (reference ``twod/solver.py:3193``): VV (TE) then HH (TM).

    The channels' systems (one per polarisation and frequency) are independent; they are
    solved together on the device worker pool, so one system's latency-bound
    factorization steps overlap another's tensor-core updates.  The result has the
    reference's co-polarised shape (``_merge_co_polarized``).
    """
    channels_by_pol = _sweep(geometry_snapshot, frequencies_ghz, elevations_deg,
                             [pol for _export, pol in _CO_POLARIZED_2D_CHANNELS], geometry_units, progress_callback,
                             0.0, compute_condition_number, max_panels, mesh_reference_ghz, abort_event,
                             quality_thresholds)
    channels = {export: channels_by_pol[pol] for export, pol in _CO_POLARIZED_2D_CHANNELS}
    failed = [f"{k}: {c['metadata']['quality_gate']['reason']}" for k, c in channels.items()
              if not c['metadata']['quality_gate']['passed']]
    if strict_quality_gate and failed:
        raise ValueError('Quality gate failed: ' + '; '.join(failed))
    return _merge_co_polarized(channels)


def _merge_co_polarized(channels, extra_metadata=None):
    """The co-polarised result in the reference's shape (``twod/solver.py:2778``
    ``_merge_co_polarized_2d_results``): ``samples`` interleave VV then HH per physical
    sample (in the VV channel's order), each row labelled with its export and internal
    polarisation; ``co_solved_samples`` keeps the two channels; the metadata carries the
    channel metadata, the VV/HH mapping and the combined quality gate."""
    co_solved = {}
    for export, internal in _CO_POLARIZED_2D_CHANNELS:
        rows = channels[export]['samples']  # this call's own records: labelled in place
        for row in rows:
            row['polarization'] = export
            row['polarization_internal'] = internal
        co_solved[export] = rows

    def key(row):
        return float(row['frequency_ghz']), float(row['theta_inc_deg']), float(row['theta_scat_deg'])

    partners = {key(row): row for row in co_solved['HH']}
    if set(partners) != {key(row) for row in co_solved['VV']}:
        raise ValueError('TE/TM 2-D solves did not return the same physical grid.')
    samples = []
    for row in co_solved['VV']:
        samples.append(row)
        samples.append(partners[key(row)])
    labels = [c[0] for c in _CO_POLARIZED_2D_CHANNELS]
    meta = {k: channels[k]['metadata'] for k in labels}
    gates = {k: dict(m.get('quality_gate', {}) or {}) for k, m in meta.items()}
    passed = all(bool(g.get('passed', False)) for g in gates.values())

    def worst(name, default=0.0):
        vals = [float(m[name]) for m in meta.values() if name in m and math.isfinite(float(m[name]))]
        return max(vals) if vals else default

    metadata = {
        'polarizations': labels,
        'polarization_internal': [c[1] for c in _CO_POLARIZED_2D_CHANNELS],
        'polarization_mapping': {'VV': 'TE', 'HH': 'TM'},
        'formulation': 'co-polarized 2-D BIE/MoM',
        'formulations': {k: m.get('formulation', '') for k, m in meta.items()},
        'panel_count_min': int(worst('panel_count_min')),
        'panel_count_max': int(worst('panel_count_max')),
        'residual_norm_max': worst('residual_norm_max'),
        'constraint_residual_norm_max': worst('constraint_residual_norm_max'),
        'condition_est_max': worst('condition_est_max', float('nan')),
        'condition_est_computed': all(bool(m.get('condition_est_computed', False)) for m in meta.values()),
        'warnings': [w for m in meta.values() for w in (m.get('warnings', []) or [])],
        'quality_gate': {'passed': passed, 'channels': gates,
                         'reason': ('Both VV<-TE and HH<-TM discrete linear-system quality gates passed' if passed
                                    else 'At least one co-polarized 2-D channel failed its quality gate')},
        'channel_metadata': meta,
        'channels': meta,
        'amplitude_version': RCS_AMPLITUDE_VERSION,
        'co_solve_shared_discretization': True,
        'linear_backend': 'gpu_grim',
        'dense_gpu_solve_count': int(sum(int(m.get('dense_gpu_solve_count', 0)) for m in meta.values())),
        'dense_cpu_solve_count': 0,
        'dense_gpu_devices': sorted({d for m in meta.values() for d in (m.get('dense_gpu_devices', []) or [])}),
        'dense_largest_system': int(worst('dense_largest_system')),
    }
    if extra_metadata:
        metadata.update(extra_metadata)
    return {
        'solver': '2d_bie_mom_rcs',
        'scattering_mode': 'monostatic',
        'amplitude_convention': RCS_AMPLITUDE_CONVENTION,
        'amplitude_version': RCS_AMPLITUDE_VERSION,
        'rcs_log_unit': 'dBke',
        'rcs_linear_quantity': 'sigma_2d',
        'polarizations': labels,
        'polarization_mapping': {'VV': 'TE', 'HH': 'TM'},
        'samples': samples,
        'co_solved_samples': co_solved,
        'metadata': metadata,
    }


# ------------------------------------------------------------------ certified (base + refined mesh)
def _certified_channels(geometry_snapshot, frequencies_ghz, elevations_deg, pols, geometry_units, progress_callback,
                        mesh_convergence_policy, max_panels, mesh_reference_ghz, cfie_alpha, abort_event,
                        quality_thresholds=None):
    """Base and refined-mesh solves of every (polarisation, frequency) system in ONE grouped
    factorization, then per polarisation and frequency the reference's certificate
    (``twod/solver.py:3663-3880``): the refined result is published only where it agrees
    with the base one within the policy, else ValueError."""
    policy = certify.validate_policy(mesh_convergence_policy)
    fine_snapshot = certify.scale_snapshot_panel_density(geometry_snapshot, policy['fine_factor'])
    # the production entry reports the condition estimate, as the reference's does
    # (twod/solver.py:3734 sets compute_condition_number for its certified pair)
    base, fine = _sweep_many([geometry_snapshot, fine_snapshot], frequencies_ghz, elevations_deg, pols,
                             geometry_units, progress_callback, cfie_alpha, True, max_panels, mesh_reference_ghz,
                             abort_event, quality_thresholds)
    out = {}
    for pol in pols:
        b, f = base[pol], fine[pol]
        b_outs, f_outs = b.pop('_outs'), f.pop('_outs')
        gates = []
        for bo, fo in zip(b_outs, f_outs):
            res = certify.certify({'samples': bo['samples'], 'metadata': b['metadata']},
                                  {'samples': fo['samples'], 'metadata': f['metadata']}, policy, bo['n'], fo['n'])
            gates.append(res['metadata']['mesh_convergence'])
        meta = dict(f['metadata'])
        qg = dict(meta.get('quality_gate', {}))
        qg.update(mesh_convergence_certified=True, certification_scope='discrete_linear_system_and_mesh_convergence')
        meta.update(quality_gate=qg, mesh_convergence=gates[0] if len(gates) == 1 else gates,
                    mesh_convergence_certified=True, certified_entry_point=True, published_mesh='fine',
                    mesh_strategy_used='global',
                    certification_phase_counters={'base': {'dense_factorization_count': len(b_outs)},
                                                  'fine': {'dense_factorization_count': len(f_outs)}})
        f['metadata'] = meta
        out[pol] = f
    return out


def solve_monostatic_rcs_2d_certified_single_polarization(
        geometry_snapshot, frequencies_ghz, elevations_deg, polarization, geometry_units="inches",
        material_base_dir=None, progress_callback=None, quality_thresholds=None, mesh_convergence_policy=None,
        max_panels=MAX_PANELS_DEFAULT, mesh_reference_ghz=None, rcs_normalization_mode="physical", cfie_alpha=0.0,
        abort_event=None, solver_method="auto", _shared_discretization_caches=None):
    """Single-polarisation solve with mesh certification (reference ``twod/solver.py:3885``):
    the base mesh and the mesh refined by the policy's ``fine_factor`` are solved together
    (one grouped factorization of all their systems) and the refined result is published
    with its ``mesh_convergence`` report, or ValueError when the two disagree."""
    pol = _canonical_user_polarization_label(polarization)
    if pol not in ('TM', 'TE'):
        raise ValueError(f'Unknown polarization {polarization!r}.')
    return _certified_channels(geometry_snapshot, frequencies_ghz, elevations_deg, [pol], geometry_units,
                               progress_callback, mesh_convergence_policy, max_panels, mesh_reference_ghz, cfie_alpha,
                               abort_event, quality_thresholds)[pol]


def solve_monostatic_rcs_2d_certified(geometry_snapshot, frequencies_ghz, elevations_deg, geometry_units="inches",
                                      material_base_dir=None, progress_callback=None, quality_thresholds=None,
                                      mesh_convergence_policy=None, max_panels=MAX_PANELS_DEFAULT,
                                      mesh_reference_ghz=None, rcs_normalization_mode="physical", abort_event=None,
                                      solver_method="auto"):
    """The reference's canonical production monostatic entry (``twod/solver.py:3979``): both
    co-polarised channels, each certified on a refined mesh; base and refined systems of
    both channels and every frequency go through one grouped factorization.  Samples VV then
    HH, as ``solve_monostatic_rcs_2d``."""
    pols = [pol for _export, pol in _CO_POLARIZED_2D_CHANNELS]
    by_pol = _certified_channels(geometry_snapshot, frequencies_ghz, elevations_deg, pols, geometry_units,
                                 progress_callback, mesh_convergence_policy, max_panels, mesh_reference_ghz, 0.0,
                                 abort_event, quality_thresholds)
    channels = {export: by_pol[pol] for export, pol in _CO_POLARIZED_2D_CHANNELS}
    return _merge_co_polarized(channels, {'mesh_convergence_certified': True, 'certified_entry_point': True,
                                          'published_mesh': 'fine',
                                          'certification_solve_order': ['base_TE', 'base_TM', 'fine_TE', 'fine_TM']})
