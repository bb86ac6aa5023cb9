"""Serving engine: same results alone and in the mix, budget admission, factor cache."""
import numpy as np
import pytest

from grim_20261007_b200 import synthetic as S

pytestmark = pytest.mark.gpu
torch = pytest.importorskip('torch')


def _requests():
    from grim_20261007_b200.serving import Request
    out = []
    for i, (n, pol) in enumerate(((192, 'TM'), (256, 'TE'), (320, 'TM'), (128, 'TE'))):
        v = S.superellipse(0.6, 0.35, 2.5 + 0.3 * i, n) if i % 2 else S.naca_symmetric(0.1 + 0.01 * i, n)
        k = 2 * np.pi / (S.polygon_perimeter(v) * 10 / n)
        out.append(Request('2d', v, k, np.arange(0.0, 360.0, 3.0 + i), pol, precision='mixed' if i < 3 else 'double'))
    out.append(Request('bor', S.sphere_generatrix(1.0, 20), 2.0, [0.0, 40.0, 90.0], precision='double', n_modes=5))
    return out


def _amps(res):
    return res['amplitude'] if 'amplitude' in res else np.concatenate([res['amp_vv'], res['amp_hh']])


def test_results_identical_alone_and_in_the_mix():
    from grim_20261007_b200.serving import ServingEngine
    alone = []
    eng = ServingEngine(slots=1)
    for r in _requests():
        alone.append(_amps(eng.submit(r).result(timeout=300)))
    eng.close()
    eng = ServingEngine(slots=4)
    futs = [eng.submit(r) for r in _requests()]
    mixed = [_amps(f.result(timeout=300)) for f in futs]
    st = eng.stats()
    eng.close()
    assert st['completed'] == len(futs) and st['max_concurrent'] >= 2
    for a, b in zip(alone, mixed):
        assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(a))
    assert st['p99_ms'] >= st['p50_ms'] > 0


def test_budget_admission_serializes_large_requests():
    from grim_20261007_b200.serving import ServingEngine
    reqs = _requests()[:3]
    budget = max(r.estimate_bytes() for r in reqs) + 1024
    eng = ServingEngine(slots=3, hbm_budget_bytes=budget, cache_bytes=0)
    for f in [eng.submit(r) for r in reqs]:
        f.result(timeout=300)
    st = eng.stats()
    eng.close()
    assert st['max_concurrent'] == 1


def test_factor_cache_reuses_resident_factors():
    from grim_20261007_b200.serving import Request, ServingEngine
    v = S.naca_symmetric(0.12, 400)
    k = 2 * np.pi / (S.polygon_perimeter(v) * 10 / 400)
    eng = ServingEngine(slots=2)
    r1 = eng.submit(Request('2d', v, k, np.arange(0, 360, 5.0), 'TE', 'mixed')).result(timeout=300)
    r2 = eng.submit(Request('2d', v, k, np.arange(0, 360, 5.0), 'TE', 'mixed')).result(timeout=300)
    r3 = eng.submit(Request('2d', v, k, [17.0, 33.0], 'TE', 'mixed')).result(timeout=300)
    eng.close()
    assert not r1['telemetry']['cache_hit'] and r2['telemetry']['cache_hit'] and r3['telemetry']['cache_hit']
    np.testing.assert_array_equal(r1['amplitude'], r2['amplitude'])
    assert eng.cache.hits >= 2
