"""The allocation-free backward error, collected last so a failure here stops nothing else.

grim_backward_error_noalloc serves callers that cannot allocate device memory when they
call it; it must give the same per-column normwise backward errors as
grim_backward_error, call after call (its fixed scratch array is reused).
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip('torch')


def _case(seed, n, m):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    x = rng.standard_normal((n, m)) + 1j * rng.standard_normal((n, m))
    b = a @ x + 1e-6 * (rng.standard_normal((n, m)) + 1j * rng.standard_normal((n, m)))
    return a, x, b


@pytest.mark.gpu
def test_noalloc_backward_error_matches_existing_entry_point_twice():
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from grim_20261007_b200 import _lib
    from grim_20261007_b200.device import context, ptr, to_device_colmajor
    ctx = context()
    for seed, n, m, c64 in ((1, 300, 17, 0), (2, 1024, 128, 1)):
        a, x, b = _case(seed, n, m)
        at = to_device_colmajor(a, torch.complex64 if c64 else torch.complex128)
        xt, bt = to_device_colmajor(x), to_device_colmajor(b)
        ref = torch.empty(m, dtype=torch.float64, device='cuda')
        got = torch.full((m,), -1.0, dtype=torch.float64, device='cuda')
        _lib.check(ctx.lib.grim_backward_error(ctx.h, n, m, ptr(at), n, c64, ptr(xt), n, ptr(bt), n, ptr(ref)))
        _lib.check(ctx.lib.grim_backward_error_noalloc(ctx.h, n, m, ptr(at), n, c64, ptr(xt), n, ptr(bt), n,
                                                       ptr(got)))
        r, g = ref.cpu().numpy(), got.cpu().numpy()
        assert np.all(r > 0)
        np.testing.assert_allclose(g, r, rtol=1e-12, atol=0)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    """Runs without a GPU: oversize requests are refused before the handle or the device is touched."""
    from grim_20261007_b200 import _lib
    lib = _lib.load()
    h = ctypes.c_void_p(1)  # size checks come before any use of the handle or the GPU
    dummy = ctypes.c_void_p(1)
    status = lib.grim_backward_error_noalloc(h, 1025, 4, dummy, 1025, 0, dummy, 1025, dummy, 1025, dummy)
    assert status == _lib.GRIM_ERR_ARGUMENT
    assert '1024' in _lib.last_error()
    status = lib.grim_backward_error_noalloc(h, 64, 129, dummy, 64, 0, dummy, 64, dummy, 64, dummy)
    assert status == _lib.GRIM_ERR_ARGUMENT
