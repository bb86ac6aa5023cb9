"""tcgen05 split-TF32 complex64 update C -= A B against a complex128 reference."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip('torch')


@pytest.mark.parametrize('m,n,k', [(64, 64, 16), (200, 150, 64), (1984, 720, 64), (37, 5, 3)])
def test_tensor_core_cgemm_matches_reference(m, n, k):
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from grim_20261007_b200 import _lib
    from grim_20261007_b200.device import context, ptr, to_device_colmajor, to_host_matrix
    ctx = context()
    rng = np.random.default_rng(m + n + k)
    a = (rng.standard_normal((m, k)) + 1j * rng.standard_normal((m, k))).astype(np.complex64)
    b = (rng.standard_normal((k, n)) + 1j * rng.standard_normal((k, n))).astype(np.complex64)
    c = (rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))).astype(np.complex64)
    ref = c.astype(np.complex128) - a.astype(np.complex128) @ b.astype(np.complex128)
    at = to_device_colmajor(a, torch.complex64)  # keep references: the kernels run asynchronously
    bt = to_device_colmajor(b, torch.complex64)
    for tc in (1, 0):
        ct = to_device_colmajor(c, torch.complex64)
        _lib.check(ctx.lib.grim_cgemm_sub(ctx.h, m, n, k, ptr(at), m, ptr(bt), k, ptr(ct), m, tc))
        got = to_host_matrix(ct).astype(np.complex128)
        scale = np.sqrt(k) * 4.0
        err = np.max(np.abs(got - ref)) / scale
        assert err < (1e-5 if tc else 2e-6), (tc, err)  # split TF32 accumulates in tensor-core FP32
