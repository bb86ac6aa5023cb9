"""The 2-D quality gate against the reference's own ``evaluate_quality_gate``
(``twod/solver.py:953``) on the cases of ``tests/golden/quality_gate.json`` (made by
``tests/golden/make_quality_gate_golden.py``)."""
import json
import math
import os

import pytest

from grim_20261007_b200.twod import quality

GOLDEN = os.path.join(os.path.dirname(__file__), 'golden', 'quality_gate.json')


def _revive(x):
    if x == 'nan':
        return float('nan')
    if isinstance(x, dict):
        return {k: _revive(v) for k, v in x.items()}
    if isinstance(x, list):
        return [_revive(v) for v in x]
    return x


def _same(a, b):
    if isinstance(a, float) and isinstance(b, float) and math.isnan(a) and math.isnan(b):
        return True
    if isinstance(a, dict) and isinstance(b, dict):
        return a.keys() == b.keys() and all(_same(a[k], b[k]) for k in a)
    if isinstance(a, list) and isinstance(b, list):
        return len(a) == len(b) and all(_same(x, y) for x, y in zip(a, b))
    return a == b


with open(GOLDEN) as _f:
    CASES = _revive(json.load(_f))['gates']


@pytest.mark.parametrize('case', CASES, ids=[str(i) for i in range(len(CASES))])
def test_quality_gate_equals_the_reference(case):
    if 'error' in case:
        with pytest.raises(ValueError) as exc:
            quality.evaluate_quality_gate(case['metadata'], case['thresholds'])
        assert str(exc.value) == case['error']
    else:
        got = quality.evaluate_quality_gate(case['metadata'], case['thresholds'])
        assert _same(got, case['result']), (got, case['result'])


def test_invalid_thresholds_fail_before_any_solve():
    from grim_20261007_b200.twod.solver import _validate_request
    with pytest.raises(ValueError, match='Unknown 2-D quality threshold'):
        _validate_request([1.0], [0.0], 0.0, False, {'residual_norm': 1.0})
    assert _validate_request([1.0], [0.0], 0.0, True, {'condition_est_max': 1e3}) == ([1.0], [0.0])
