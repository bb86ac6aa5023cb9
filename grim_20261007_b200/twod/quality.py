"""Numeric quality gate of a 2-D solve, restating the reference's ``evaluate_quality_gate``
(``twod/solver.py:953-1100``): the same thresholds, defaults, validation, violations and
reason text, evaluated on this package's channel metadata.

Thresholds (defaults): ``residual_norm_max`` 1e-6 (the largest per-sample linear
residual), ``constraint_residual_norm_max`` 1e-8 (junction constraints; none are applied on
this path), ``condition_est_max`` 1e6 (checked only when the condition number was
computed), ``warnings_max`` 10.  Unknown threshold names, negative or non-finite limits and a
non-integer ``warnings_max`` raise ``ValueError``, as in the reference.
"""
from __future__ import annotations

import math

DEFAULTS = {
    'residual_norm_max': 1.0e-6,
    'constraint_residual_norm_max': 1.0e-8,
    'condition_est_max': 1.0e6,
    'warnings_max': 10,
}


def merged_thresholds(thresholds=None):
    """The gate's limits: defaults overridden by ``thresholds`` (validated)."""
    merged = dict(DEFAULTS)
    if thresholds:
        supplied = dict(thresholds)
        unknown = sorted(set(supplied) - set(DEFAULTS))
        if unknown:
            raise ValueError('Unknown 2-D quality threshold field(s): ' + ', '.join(str(k) for k in unknown))
        merged.update(supplied)
    limits = {}
    for key in ('residual_norm_max', 'constraint_residual_norm_max', 'condition_est_max'):
        value = float(merged[key])
        if not math.isfinite(value) or value < 0.0:
            raise ValueError('2-D residual and condition quality thresholds must be finite non-negative values.')
        limits[key] = value
    try:
        w = float(merged['warnings_max'])
    except (TypeError, ValueError, OverflowError) as exc:
        raise ValueError('warnings_max must be a finite non-negative integer.') from exc
    if not math.isfinite(w) or w < 0.0 or not w.is_integer():
        raise ValueError('warnings_max must be a finite non-negative integer.')
    limits['warnings_max'] = int(w)
    return limits


def _as_float(value):
    try:
        return float(value) if value is not None else float('nan')
    except (TypeError, ValueError):
        return float('nan')


def evaluate_quality_gate(metadata, thresholds=None):
    """Gate verdict for one channel's metadata: dict(passed, thresholds, values, violations,
    certification_scope, mesh_convergence_certified, reason)."""
    limits = merged_thresholds(thresholds)
    residual = _as_float(metadata.get('residual_norm_max'))
    try:
        nonfinite = int(metadata.get('residual_nonfinite_count', 0))
    except (TypeError, ValueError, OverflowError):
        nonfinite = -1
    constraint = float(metadata.get('constraint_residual_norm_max', 0.0) or 0.0)
    condition = _as_float(metadata.get('condition_est_max'))
    if 'condition_est_computed' in metadata:
        computed = bool(metadata.get('condition_est_computed'))
    else:
        computed = math.isfinite(condition)
    warnings_count = len(list(metadata.get('warnings', []) or []))

    violations = []
    if not math.isfinite(residual) or residual > limits['residual_norm_max']:
        violations.append(f"residual_norm_max={residual:.6g} exceeds limit {limits['residual_norm_max']:.6g}")
    if nonfinite != 0:
        violations.append(f'residual_nonfinite_count={nonfinite} must be zero' if nonfinite > 0
                          else 'residual_nonfinite_count is missing a valid non-negative integer value')
    if bool(metadata.get('junction_constraints_applied', False)) and (
            not math.isfinite(constraint) or constraint > limits['constraint_residual_norm_max']):
        violations.append(f"constraint_residual_norm_max={constraint:.6g} exceeds limit "
                          f"{limits['constraint_residual_norm_max']:.6g}")
    if computed and (not math.isfinite(condition) or condition > limits['condition_est_max']):
        violations.append(f"condition_est_max={condition:.6g} exceeds limit {limits['condition_est_max']:.6g}")
    if warnings_count > limits['warnings_max']:
        violations.append(f"warnings_count={warnings_count} exceeds limit {limits['warnings_max']}")
    if violations:
        reason = '; '.join(violations)
    else:
        reason = ('discrete linear-system quality thresholds satisfied; '
                  + ('condition number was not requested; ' if not computed else '')
                  + 'mesh convergence is separately certified by the production workflow')
    return {
        'passed': not violations,
        'thresholds': dict(limits),
        'values': {
            'residual_norm_max': residual,
            'residual_nonfinite_count': nonfinite,
            'constraint_residual_norm_max': constraint,
            'condition_est_max': condition,
            'condition_est_computed': computed,
            'warnings_count': warnings_count,
        },
        'violations': violations,
        'certification_scope': ('discrete_linear_system_residual_and_condition' if computed
                                else 'discrete_linear_system_residual_only'),
        'mesh_convergence_certified': bool(metadata.get('mesh_convergence_certified', False)),
        'reason': reason,
    }
