"""Far-field Galerkin block quadrature (reference twod/assembly/native/far.c ghost_far_block):
the CPU restatement against the reference's own outputs, and the library's exports."""
import ctypes
import os

import numpy as np
import pytest

from oracle import farblock as F

GOLDEN = os.path.join(os.path.dirname(__file__), 'golden', 'far_block.npz')
REF_LIB = os.path.join(os.path.dirname(os.path.dirname(__file__)), 'oracle', '_ref', 'libghost_far_ref.so')


def case(g, name):
    keys = ('obs_pts', 'src_pts', 'qw', 'phi', 'obs_norm', 'src_norm', 'far')
    return {key: g[f'{name}_{key}'] for key in keys}, complex(g[f'{name}_k']), g[f'{name}_bounds'], \
        g[f'{name}_power'], float(g[f'{name}_upper'])


@pytest.mark.parametrize('name', ['w2', 'w3'])
@pytest.mark.parametrize('ond', [0, 1])
def test_restatement_matches_reference_outputs(name, ond):
    """Inside the table the restatement reproduces the reference bit for bit; pairs that
    reach the large-argument expansion agree to 1e-13 (cmath vs the C library)."""
    g = np.load(GOLDEN)
    inp, k, bounds, power, upper = case(g, name)
    got = F.far_block(inp['obs_pts'], inp['src_pts'], inp['qw'], inp['phi'], inp['obs_norm'], inp['src_norm'],
                      inp['far'], ond, 1, 1, 1, k, bounds, power)
    inside = F.in_table(inp['obs_pts'], inp['src_pts'], inp['far'], upper)
    outside = inp['far'].astype(bool) & ~inside
    assert inside.sum() > 20 and outside.sum() > 5
    for acc, tag in zip(got, ('s', 'k', 'kt')):
        ref = g[f'{name}_ond{ond}_{tag}']
        assert np.array_equal(acc[:, inside], ref[:, inside]), tag
        scale = np.abs(ref[:, outside]).max()
        assert np.max(np.abs(acc[:, outside] - ref[:, outside])) <= 1e-13 * scale, tag
        assert np.all(acc[:, ~inp['far'].astype(bool)] == 0)


def test_restatement_reports_below_table():
    g = np.load(GOLDEN)
    inp, k, bounds, power, _upper = case(g, 'w2')
    src = inp['src_pts'].copy()
    i, j = np.argwhere(inp['far'])[0]
    src[j] = inp['obs_pts'][i]  # coincident points: the distance is clamped to 1e-12
    b2 = bounds.copy()
    b2[0] = 1e-6  # ... which lies below a table that starts at 1e-6
    assert F.far_block(inp['obs_pts'], src, inp['qw'], inp['phi'], inp['obs_norm'], inp['src_norm'], inp['far'],
                       0, 1, 0, 0, k, b2, power) is None


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason='reference far.c not built here (oracle/build_ref.py)')
def test_restatement_matches_reference_library_on_a_fresh_case():
    g = np.load(GOLDEN)
    inp, k, bounds, power, upper = case(g, 'w2')
    rng = np.random.default_rng(5)
    obs = inp['obs_pts'] + 0.01 * rng.standard_normal(inp['obs_pts'].shape)
    lib = ctypes.CDLL(REF_LIB)
    from tests.golden.make_far_golden import reference_far
    status, ref = reference_far(lib, np.ascontiguousarray(obs), inp['src_pts'], inp['qw'], inp['phi'],
                                inp['obs_norm'], inp['src_norm'], inp['far'], 1, 1, 1, 0, k, bounds, power)
    assert status == 0
    got = F.far_block(obs, inp['src_pts'], inp['qw'], inp['phi'], inp['obs_norm'], inp['src_norm'], inp['far'], 1,
                      1, 1, 0, k, bounds, power)
    inside = F.in_table(obs, inp['src_pts'], inp['far'], upper)
    for acc, r in zip(got[:2], ref[:2]):
        assert np.array_equal(acc[:, inside], r[:, inside])
