"""Generate ``quality_gate.json``: the reference's own 2-D quality gate
(``twod/solver.py:953`` ``evaluate_quality_gate``) on seeded metadata/threshold cases, and its
equilibrated condition estimate (``twod/solver.py:529`` ``_equilibrated_condition_from_lu``,
SciPy LU) on the seeded complex matrices of ``matrices()`` (recreated by the tests, not
stored), with their exact equilibrated 1-norm condition numbers.

Run in the build container (the reference tree is not present on GPU machines):

    python tests/golden/make_quality_gate_golden.py <reference root>

(or with the root in GRIM_REFERENCE_ROOT).  The reference package is imported from its tree
without writing into it (no bytecode).
"""
from __future__ import annotations

import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def gate_cases():
    """(metadata, thresholds) pairs covering every violation and the threshold validation."""
    nan = float('nan')
    return [
        ({'residual_norm_max': 1e-9}, None),
        ({'residual_norm_max': 2e-6}, None),
        ({'residual_norm_max': 2e-6}, {'residual_norm_max': 1e-5}),
        ({'residual_norm_max': nan}, None),
        ({'residual_norm_max': 1e-9, 'residual_nonfinite_count': 3}, None),
        ({'residual_norm_max': 1e-9, 'residual_nonfinite_count': 'x'}, None),
        ({'residual_norm_max': 1e-9, 'condition_est_max': 5e6, 'condition_est_computed': True}, None),
        ({'residual_norm_max': 1e-9, 'condition_est_max': 5e6, 'condition_est_computed': False}, None),
        ({'residual_norm_max': 1e-9, 'condition_est_max': 5e6}, None),
        ({'residual_norm_max': 1e-9, 'condition_est_max': 5e6, 'condition_est_computed': True},
         {'condition_est_max': 1e7}),
        ({'residual_norm_max': 1e-9, 'condition_est_max': nan, 'condition_est_computed': True}, None),
        ({'residual_norm_max': 1e-9, 'warnings': ['a'] * 11}, None),
        ({'residual_norm_max': 1e-9, 'warnings': ['a'] * 11}, {'warnings_max': 20}),
        ({'residual_norm_max': 1e-9, 'junction_constraints_applied': True,
          'constraint_residual_norm_max': 1e-7}, None),
        ({'residual_norm_max': 1e-9, 'mesh_convergence_certified': True}, None),
        ({'residual_norm_max': 1e-9}, {'bogus': 1}),
        ({'residual_norm_max': 1e-9}, {'residual_norm_max': -1.0}),
        ({'residual_norm_max': 1e-9}, {'warnings_max': 2.5}),
    ]


def matrices():
    rng = np.random.default_rng(20261204)
    out = []
    for n, spread in ((6, 1.0), (40, 1.0), (150, 1e4), (300, 1e2)):
        a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        a *= np.exp(rng.uniform(0.0, np.log(spread), n))[:, None]  # badly scaled rows
        a += np.diag(np.full(n, 0.5 * n))
        out.append(a)
    return out


def exact_equilibrated_cond1(a):
    r = np.max(np.abs(a), axis=1)
    r = np.where(r > 0, r, 1.0)
    e = np.abs(a) / r[:, None]
    c = np.max(e, axis=0)
    c = np.where(c > 0, c, 1.0)
    b = a / r[:, None] / c[None, :]
    return float(np.linalg.norm(b, 1) * np.linalg.norm(np.linalg.inv(b), 1))


def _jsonable(x):
    if isinstance(x, float) and not math.isfinite(x):
        return repr(x)
    if isinstance(x, dict):
        return {k: _jsonable(v) for k, v in x.items()}
    if isinstance(x, (list, tuple)):
        return [_jsonable(v) for v in x]
    return x


def main(reference_root):
    sys.dont_write_bytecode = True
    sys.path.insert(0, os.path.join(reference_root, 'tools', 'GHOST'))
    import scipy.linalg as sla
    import ghost_backend.twod.solver as rcs
    gates = []
    for meta, thr in gate_cases():
        try:
            res = rcs.evaluate_quality_gate(dict(meta), thresholds=thr)
            gates.append({'metadata': meta, 'thresholds': thr, 'result': res})
        except ValueError as exc:
            gates.append({'metadata': meta, 'thresholds': thr, 'error': str(exc)})
    conds = []
    for a in matrices():
        lu, piv = sla.lu_factor(a)
        conds.append({'n': int(a.shape[0]),
                      'reference_estimate': float(rcs._equilibrated_condition_from_lu(a, lu, piv)),
                      'exact': exact_equilibrated_cond1(a)})
    with open(os.path.join(HERE, 'quality_gate.json'), 'w') as f:
        json.dump(_jsonable({'gates': gates, 'conditions': conds}), f)


if __name__ == '__main__':
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('GRIM_REFERENCE_ROOT')
    if not root:
        raise SystemExit('usage: make_quality_gate_golden.py <reference root> (or GRIM_REFERENCE_ROOT)')
    main(root)
