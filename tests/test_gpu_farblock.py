"""GPU far-field Galerkin blocks (grim_far_block / ghost_far_block) against the reference's
own outputs (tests/golden/far_block.npz, made by its compiled far.c) and, where it was
built here, the reference library itself on larger inputs."""
import ctypes
import os

import numpy as np
import pytest

from oracle import farblock as F

pytestmark = pytest.mark.gpu

torch = pytest.importorskip('torch')

GOLDEN = os.path.join(os.path.dirname(__file__), 'golden', 'far_block.npz')
REF_LIB = os.path.join(os.path.dirname(os.path.dirname(__file__)), 'oracle', '_ref', 'libghost_far_ref.so')
KEYS = ('obs_pts', 'src_pts', 'qw', 'phi', 'obs_norm', 'src_norm', 'far')


class Table:
    def __init__(self, bounds, power):
        self.bounds, self.normalized_power = bounds, power


def case(g, name):
    return ({key: np.ascontiguousarray(g[f'{name}_{key}']) for key in KEYS}, complex(g[f'{name}_k']),
            g[f'{name}_bounds'], g[f'{name}_power'], float(g[f'{name}_upper']))


def device_far(inp, ond, k, bounds, power, want=(1, 1, 1)):
    """grim_far_block on device copies of the inputs."""
    from grim_20261007_b200.device import context
    ctx = context()
    d = {key: torch.as_tensor(v, device='cuda') for key, v in inp.items()}
    mb, q = inp['obs_pts'].shape[:2]
    nb, width = inp['src_pts'].shape[0], inp['phi'].shape[1]
    db = torch.as_tensor(bounds, device='cuda')
    dc = torch.as_tensor(np.ascontiguousarray(power).view(np.float64), device='cuda')
    accs = [torch.zeros((width * width, mb, nb), dtype=torch.complex128, device='cuda') if w else None for w in
            (want[0], want[1], want[1] and want[2])]
    p = [ctypes.c_void_p(d[key].data_ptr()) for key in KEYS]
    status = ctx.lib.grim_far_block(ctx.h, mb, nb, q, width, *p, ond, want[0], want[1], want[2], k.real, k.imag,
                                    len(bounds) - 1, ctypes.c_void_p(db.data_ptr()), power.shape[1] - 1,
                                    ctypes.c_void_p(dc.data_ptr()),
                                    *(None if a is None else ctypes.c_void_p(a.data_ptr()) for a in accs))
    return status, [None if a is None else a.cpu().numpy() for a in accs]


@pytest.mark.parametrize('name', ['w2', 'w3'])
@pytest.mark.parametrize('ond', [0, 1])
@pytest.mark.parametrize('entry', ['device', 'host'])
def test_far_block_matches_reference_outputs(name, ond, entry):
    """Pairs inside the kernel table: bitwise the reference's sums.  Pairs reaching the
    large-argument expansion: 1e-13 (CUDA's exp/sincos vs the C library's)."""
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    g = np.load(GOLDEN)
    inp, k, bounds, power, upper = case(g, name)
    if entry == 'device':
        status, got = device_far(inp, ond, k, bounds, power)
        assert status == 0
    else:
        from grim_20261007_b200.twod.farblock import far_block
        got = far_block(Table(bounds, power), k, inp['obs_pts'], inp['src_pts'], inp['qw'], inp['phi'],
                        inp['obs_norm'], inp['src_norm'], inp['far'], ond, True, True, True)
    inside = F.in_table(inp['obs_pts'], inp['src_pts'], inp['far'], upper)
    outside = inp['far'].astype(bool) & ~inside
    for acc, tag in zip(got, ('s', 'k', 'kt')):
        ref = g[f'{name}_ond{ond}_{tag}']
        assert np.array_equal(acc[:, inside], ref[:, inside]), \
            f'{tag}: max |gpu - ref| inside the table {np.max(np.abs(acc[:, inside] - ref[:, inside])):.3g}'
        assert np.max(np.abs(acc[:, outside] - ref[:, outside])) <= 1e-13 * np.abs(ref[:, outside]).max(), tag
        assert np.all(acc[:, ~inp['far'].astype(bool)] == 0)


def test_far_block_wider_bases_and_partial_outputs():
    """Width 5 (the generic path) and S alone / K without the mirrored block, against the
    restatement."""
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    g = np.load(GOLDEN)
    inp, k, bounds, power, upper = case(g, 'w2')
    rng = np.random.default_rng(3)
    q = inp['qw'].shape[0]
    inp['phi'] = np.ascontiguousarray(rng.uniform(-1, 1, (q, 5)))
    inside = F.in_table(inp['obs_pts'], inp['src_pts'], inp['far'], upper)
    ref = F.far_block(*(inp[key] for key in KEYS), 0, 1, 1, 0, k, bounds, power)
    status, got = device_far(inp, 0, k, bounds, power, want=(1, 1, 0))
    assert status == 0 and got[2] is None
    for acc, r in zip(got[:2], ref[:2]):
        assert np.array_equal(acc[:, inside], r[:, inside])
    status, got = device_far(inp, 1, k, bounds, power, want=(1, 0, 0))
    ref = F.far_block(*(inp[key] for key in KEYS), 1, 1, 0, 0, k, bounds, power)
    assert status == 0 and np.array_equal(got[0][:, inside], ref[0][:, inside])


def test_far_block_status_codes():
    """2 when a far distance falls below the table (the caller's fallback), 3 on bad
    arguments, as the reference's far.c returns."""
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from grim_20261007_b200 import _lib
    g = np.load(GOLDEN)
    inp, k, bounds, power, _upper = case(g, 'w2')
    b2 = bounds.copy()
    b2[0] = 1e-6
    i, j = np.argwhere(inp['far'])[0]
    inp['src_pts'] = inp['src_pts'].copy()
    inp['src_pts'][j] = inp['obs_pts'][i]
    status, _ = device_far(inp, 0, k, b2, power)
    assert status == 2
    from grim_20261007_b200.twod.farblock import far_block
    assert far_block(Table(b2, power), k, *(inp[key] for key in KEYS), 0, True, False, False) is None
    lib = _lib.load()
    assert lib.ghost_far_block(1, 1, 0, 2, *([None] * 7), 0, 1, 0, 0, 1.0, 0.0, 1, None, 1, None, None, None,
                               None) == 3


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason='reference far.c not built (oracle/build_ref.py)')
def test_far_block_matches_reference_library_on_a_large_tile():
    """A 160 x 150 element tile (24,000 pairs, 5 x 5 points): bitwise equal to the
    reference's compiled kernel on every pair inside the table."""
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from tests.golden.make_far_golden import geometry, reference_far
    g = np.load(GOLDEN)
    _inp, k, bounds, power, upper = case(g, 'w2')
    rng = np.random.default_rng(11)
    obs, _s, qw, phi, on, centre, length = geometry(rng, 160, 0.5, 5, 2)
    _o, src, _q, _p, sn, _c, _l = geometry(rng, 150, 0.5, 5, 2, far_out=10, far_distance=1.5)
    dcent = np.linalg.norm(centre[:, None, :] - src.mean(axis=1)[None, :, :], axis=-1)
    far = np.ascontiguousarray((dcent > 3 * np.median(length)).astype(np.uint8))
    inp = dict(zip(KEYS, (obs, src, qw, phi, on, sn, far)))
    inp = {key: np.ascontiguousarray(v) for key, v in inp.items()}
    status, ref = reference_far(ctypes.CDLL(REF_LIB), *(inp[key] for key in KEYS), 1, 1, 1, 1, k, bounds, power)
    assert status == 0
    status, got = device_far(inp, 1, k, bounds, power)
    assert status == 0
    inside = F.in_table(obs, src, far, upper)
    outside = far.astype(bool) & ~inside
    assert inside.sum() > 10000
    for acc, r in zip(got, ref):
        assert np.array_equal(acc[:, inside], r[:, inside])
        if outside.any():
            assert np.max(np.abs(acc[:, outside] - r[:, outside])) <= 1e-13 * np.abs(r[:, outside]).max()


def test_far_block_width_one_single_point():
    """Width 1 and one quadrature point (the generic kernel) against the restatement."""
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    g = np.load(GOLDEN)
    inp, k, bounds, power, upper = case(g, 'w2')
    inp['obs_pts'] = np.ascontiguousarray(inp['obs_pts'][:, :1])
    inp['src_pts'] = np.ascontiguousarray(inp['src_pts'][:, :1])
    inp['qw'] = np.ones(1)
    inp['phi'] = np.ones((1, 1))
    inside = F.in_table(inp['obs_pts'], inp['src_pts'], inp['far'], upper)
    ref = F.far_block(*(inp[key] for key in KEYS), 1, 1, 1, 1, k, bounds, power)
    status, got = device_far(inp, 1, k, bounds, power)
    assert status == 0
    for acc, r in zip(got, ref):
        assert np.array_equal(acc[:, inside], r[:, inside])
