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


@pytest.mark.parametrize('n,nrhs', [(700, 150), (1024, 300), (1300, 200)])
def test_mixed_solve_on_packed_block_panels(n, nrhs):
    """Wide right-hand sides take the packed-panel complex64 solve; refinement still reaches FP64."""
    import ctypes
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from grim_20261007_b200 import _lib
    from grim_20261007_b200.device import context, ptr, to_device_colmajor, to_host_matrix
    ctx = context()
    rng = np.random.default_rng(n)
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    b = rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs))
    at = to_device_colmajor(a, torch.complex128)
    bt = to_device_colmajor(b, torch.complex128)
    info, st = ctypes.c_int(-1), _lib.GrimSolveInfo()
    _lib.check(ctx.lib.grim_zgesv_mixed(ctx.h, n, nrhs, ptr(at), n, None, 0, ptr(bt), n, _lib.PREC_MIXED, 1e-12, 10,
                                        ctypes.byref(info), ctypes.byref(st)))
    x = to_host_matrix(bt)
    ref = np.linalg.solve(a, b)
    assert info.value == 0
    assert np.max(np.abs(x - ref)) <= 1e-10 * np.max(np.abs(ref)), st.as_dict()
    assert st.initial_backward_error < 1e-4 and st.refinement_steps >= 1, st.as_dict()


@pytest.mark.parametrize('n,nrhs', [(1100, 200), (2048, 720)])
def test_mixed_solve_without_row_interchanges(n, nrhs):
    """A diagonally dominant system factors on the certified path (no row interchanges, a
    partial last panel block at n = 1100); the packed-panel solve and the refinement still
    reach FP64."""
    import ctypes
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from grim_20261007_b200 import _lib
    from grim_20261007_b200.device import context, ptr, to_device_colmajor, to_host_matrix
    ctx = context()
    rng = np.random.default_rng(n + 1)
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)) + 4.0 * np.sqrt(n) * np.eye(n)
    b = rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs))
    at = to_device_colmajor(a, torch.complex128)
    bt = to_device_colmajor(b, torch.complex128)
    info, st = ctypes.c_int(-1), _lib.GrimSolveInfo()
    _lib.check(ctx.lib.grim_zgesv_mixed(ctx.h, n, nrhs, ptr(at), n, None, 0, ptr(bt), n, _lib.PREC_MIXED, 1e-12, 10,
                                        ctypes.byref(info), ctypes.byref(st)))
    x = to_host_matrix(bt)
    ref = np.linalg.solve(a, b)
    assert info.value == 0 and st.pivoted_panels == 0, st.as_dict()
    assert np.max(np.abs(x - ref)) <= 1e-10 * np.max(np.abs(ref)), st.as_dict()


@pytest.mark.parametrize('n,nrhs,complex64', [(300, 37, True), (300, 37, False), (1024, 130, True)])
def test_integer_slice_residual_matches_fp64(n, nrhs, complex64):
    """R = B - A X on the int8 tensor cores agrees with an FP64 residual: to FP64 accuracy with 8
    slices, within the truncation of 7 (about 6e-15 of max |A||X|) and 6 slices (about 1e-12)."""
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from grim_20261007_b200 import _lib
    from grim_20261007_b200.device import context, ptr, to_device_colmajor, to_host_matrix
    ctx = context()
    rng = np.random.default_rng(n + nrhs)
    a = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) * np.exp(2 * rng.standard_normal((n, 1)))
    if complex64:
        a = a.astype(np.complex64).astype(np.complex128)
    x = (rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs))) * np.exp(rng.standard_normal(nrhs))
    x[:, 5] = 0.0
    b = a @ x + 1e-9 * (rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs)))
    at = to_device_colmajor(a, torch.complex64 if complex64 else torch.complex128)
    xt, bt = to_device_colmajor(x, torch.complex128), to_device_colmajor(b, torch.complex128)
    out = {}
    for slices in (8, 7, 6, 0):
        rt = to_device_colmajor(np.zeros((n, nrhs)), torch.complex128)
        _lib.check(ctx.lib.grim_residual(ctx.h, n, nrhs, ptr(at), n, int(complex64), ptr(xt), n, ptr(bt), n, ptr(rt), n,
                                         slices))
        out[slices] = to_host_matrix(rt)
    ref = b - a @ x
    bound = 2e-14 * (np.abs(a) @ np.abs(x)).max()
    assert np.max(np.abs(out[8] - ref)) <= bound
    assert np.max(np.abs(out[0] - ref)) <= bound
    assert np.max(np.abs(out[7] - ref)) <= 50 * bound  # 7 slices: about 6e-15 of max |A||X|
    assert np.max(np.abs(out[6] - ref)) <= 400 * bound  # 6 slices: 2^7 times the 7-slice truncation


def test_integer_slice_residual_propagates_nonfinite():
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from grim_20261007_b200 import _lib
    from grim_20261007_b200.device import context, ptr, to_device_colmajor, to_host_matrix
    ctx = context()
    rng = np.random.default_rng(9)
    n, nrhs = 256, 20
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    x = rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs))
    x[17, 3] = np.nan
    b = np.ones((n, nrhs), complex)
    at, xt, bt = (to_device_colmajor(v, torch.complex128) for v in (a, x, b))
    rt = to_device_colmajor(np.zeros((n, nrhs)), torch.complex128)
    _lib.check(ctx.lib.grim_residual(ctx.h, n, nrhs, ptr(at), n, 0, ptr(xt), n, ptr(bt), n, ptr(rt), n, 8))
    r = to_host_matrix(rt)
    assert np.all(np.isnan(r[:, 3]))
    assert np.all(np.isfinite(np.delete(r, 3, axis=1)))


def test_backward_error_stopping_mode():
    """GRIM_PREC_MIXED_BERR stops on the normwise backward error; GRIM_PREC_MIXED on the relative residual."""
    import ctypes
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from grim_20261007_b200 import _lib
    from grim_20261007_b200.device import context, ptr, to_device_colmajor, to_host_matrix
    ctx = context()
    rng = np.random.default_rng(5)
    n, nrhs = 600, 64
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)) + 8 * np.sqrt(n) * np.eye(n)
    b = rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs))
    at = to_device_colmajor(a, torch.complex128)
    for mode in (_lib.PREC_MIXED, _lib.PREC_MIXED_BERR):
        bt = to_device_colmajor(b, torch.complex128)
        info, st = ctypes.c_int(-1), _lib.GrimSolveInfo()
        _lib.check(ctx.lib.grim_zgesv_mixed(ctx.h, n, nrhs, ptr(at), n, None, 0, ptr(bt), n, mode, 1e-10, 10,
                                            ctypes.byref(info), ctypes.byref(st)))
        x = to_host_matrix(bt)
        r = a @ x - b
        berr = np.max(np.abs(r), axis=0) / (np.max(np.sum(np.abs(a), axis=1)) * np.max(np.abs(x), axis=0)
                                            + np.max(np.abs(b), axis=0))
        relres = np.max(np.abs(r), axis=0) / np.max(np.abs(b), axis=0)
        if mode == _lib.PREC_MIXED_BERR:
            assert np.max(berr) <= 1e-10 * 1.01 and st.backward_error <= 1e-10, st.as_dict()
        else:
            assert np.max(relres) <= 1e-10 * 1.01, st.as_dict()


def test_autotuner_times_every_candidate_and_keeps_results(tmp_path, monkeypatch):
    """The tuner times each tile-shape pair on a seeded system and the chosen shapes give the same solution."""
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from grim_20261007_b200 import synthetic as S, tuning
    from grim_20261007_b200.device import context
    from grim_20261007_b200.twod import geometry as geo, operators as ops
    monkeypatch.setenv('GRIM_TUNING_CACHE', str(tmp_path / 'tuning.json'))
    monkeypatch.setattr(tuning, '_table', None)
    ctx = context()
    entry = tuning.tune_dense(640, 200, ctx=ctx, reps=1)
    ncand = len(tuning.CANDIDATES['solve_bn']) * len(tuning.CANDIDATES['gs_block'])
    assert len(entry['timings_ms']) == ncand and entry['choice']['solve_bn'] in (64, 128)
    assert tuning.lookup(ctx.device_name, 640, 200)['choice'] == entry['choice']
    v, k, _f, _t = S.airfoil_case(0, 640)
    body = ops.DeviceBody(geo.panel_geometry([v]), None)
    ang = torch.as_tensor(np.arange(200) * 1.8, device='cuda')
    z32 = ops.fill(body, k, 'TM', complex64=True)
    b0 = ops.rhs(body, k, 'TM', ang)
    xs = []
    for shapes in ((64, 256), (128, 512)):
        tuning.set_handle(ctx, *shapes)
        b = b0.clone()
        ops.solve_inplace(None, b, 'mixed', tol=1e-10, z32=z32, stop='berr', tuned=False)
        xs.append(b.cpu().numpy())
    tuning.set_handle(ctx, 0, 0)
    np.testing.assert_allclose(xs[0], xs[1], rtol=1e-8, atol=1e-8 * np.max(np.abs(xs[1])))
