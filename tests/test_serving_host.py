"""Host logic of the serving engine (no GPU): the factor cache's pinning and eviction and the
admission rule that counts the cache against the device budget."""
from grim_20261007_b200.serving.engine import FactorCache, admission_fits


def test_pinned_entries_survive_eviction_and_the_cache_stays_within_capacity():
    c = FactorCache(100)
    c.put('a', {}, 40)
    c.put('b', {}, 40)
    assert c.used == 80
    assert c.pin('a') and not c.pin('zz')
    c.put('c', {}, 40)            # evicts b (a is pinned although older)
    assert set(c.items) == {'a', 'c'} and c.used == 80
    c.put('d', {}, 70)            # would need a evicted: refused, capacity kept
    assert set(c.items) == {'a', 'c'} and c.used == 80
    assert c.shrink_to(50) and set(c.items) == {'a'} and c.used == 40
    assert not c.shrink_to(0)     # a is still pinned
    c.unpin('a')
    assert c.shrink_to(0) and c.used == 0 and not c.items


def test_admission_counts_the_cache_against_the_budget():
    assert admission_fits(in_use=50, est=30, cache_used=20, budget=100, running=1)
    assert not admission_fits(in_use=50, est=30, cache_used=21, budget=100, running=1)
    # alone on the device a request always runs (the budget only orders concurrent ones)
    assert admission_fits(in_use=0, est=500, cache_used=90, budget=100, running=0)
