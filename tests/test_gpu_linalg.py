"""GPU dense LU / solve parity through the C ABI (LAPACK getrf/getrs via scipy as the oracle)."""
import ctypes
import os

import numpy as np
import pytest
import scipy.linalg as sla

from tests.conftest import GOLDEN

pytestmark = pytest.mark.gpu

torch = pytest.importorskip('torch')


@pytest.fixture(scope='module')
def ctx():
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from grim_20261007_b200.device import context
    return context()


def _dev(a, dtype=None):
    from grim_20261007_b200.device import to_device_colmajor
    return to_device_colmajor(a, dtype=dtype or torch.complex128)


def _host(t):
    from grim_20261007_b200.device import to_host_matrix
    return to_host_matrix(t)


def _rand(n, m, seed, dominant=False):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((n, m)) + 1j * rng.standard_normal((n, m))
    if dominant:
        a += np.diag(np.full(n, 4.0 * n))
    return a


def _getrf(ctx, a, complex64=False, pivot=0):
    from grim_20261007_b200 import _lib
    from grim_20261007_b200.device import ptr
    n = a.shape[0]
    t = _dev(a, torch.complex64 if complex64 else torch.complex128)
    ipiv = torch.zeros(n, dtype=torch.int32, device='cuda')
    info = ctypes.c_int(-1)
    fn = ctx.lib.grim_cgetrf if complex64 else ctx.lib.grim_zgetrf
    _lib.check(ctx.lib.grim_set_tuning(ctx.h, _lib.TUNE_PIVOT, pivot))
    try:
        _lib.check(fn(ctx.h, n, ptr(t), n, ptr(ipiv), ctypes.byref(info)))
    finally:
        ctx.lib.grim_set_tuning(ctx.h, _lib.TUNE_PIVOT, _lib.PIVOT_CERTIFIED)
    return t, ipiv, info.value


@pytest.mark.parametrize('n', [1, 7, 64, 97, 200, 333, 1100, 2048, 2100, 3500])
def test_partial_pivoting_getrf_matches_lapack(ctx, n):
    """Partial pivoting on a thread-block cluster: LAPACK's pivots and factors, for cluster
    sizes 1 to 16, panels of up to 16 x 128 rows in registers (n = 2048 fills all 16 CTAs)
    and taller panels in shared memory (n = 2100, 3500; 3500 also past a CTA's shared
    memory)."""
    from grim_20261007_b200 import _lib
    a = _rand(n, n, 300 + n)
    t, ipiv, info = _getrf(ctx, a, pivot=_lib.PIVOT_PARTIAL)
    lu_ref, piv_ref = sla.lu_factor(a)
    assert info == 0
    np.testing.assert_array_equal(ipiv.cpu().numpy(), piv_ref + 1)
    lu = _host(t)
    assert np.max(np.abs(lu - lu_ref)) <= 1e-10 * max(1.0, np.max(np.abs(lu_ref)))


def _lapack_perm(ipiv):
    """Row order of LAPACK's sequential interchanges (1-based ipiv)."""
    perm = np.arange(len(ipiv))
    for i, p in enumerate(ipiv - 1):
        perm[[i, p]] = perm[[p, i]]
    return perm


def test_partial_pivoting_cgetrf_large_is_a_partial_pivoting_lu(ctx):
    """complex64 at n = 2048 (16 CTAs of 128 register-resident rows): LAPACK's FP32 blocked
    order rounds differently, so near-ties may pick other rows; the factors must still be a
    partial-pivoting LU of A: P A = L U to FP32 accuracy, and no multiplier larger than the
    pivot search allows (|re| + |im| of the pivot is the column's largest, so |l| <= sqrt 2)."""
    from grim_20261007_b200 import _lib
    n = 2048
    a = _rand(n, n, 4242).astype(np.complex64)
    t, ipiv, info = _getrf(ctx, a, complex64=True, pivot=_lib.PIVOT_PARTIAL)
    assert info == 0
    lu = _host(t).astype(np.complex128)
    low = np.tril(lu, -1) + np.eye(n)
    up = np.triu(lu)
    assert np.max(np.abs(low)) <= np.sqrt(2.0) * (1.0 + 1e-5)
    pa = a.astype(np.complex128)[_lapack_perm(ipiv.cpu().numpy())]
    assert np.max(np.abs(pa - low @ up)) <= 1e-4 * np.max(np.abs(a))


@pytest.mark.parametrize('n', [160, 700])
def test_partial_pivoting_cgetrf_matches_lapack(ctx, n):
    from grim_20261007_b200 import _lib
    a = _rand(n, n, 31 + n).astype(np.complex64)
    t, ipiv, info = _getrf(ctx, a, complex64=True, pivot=_lib.PIVOT_PARTIAL)
    lu_ref, piv_ref = sla.lu_factor(a)
    assert info == 0
    np.testing.assert_array_equal(ipiv.cpu().numpy(), piv_ref + 1)
    assert np.max(np.abs(_host(t) - lu_ref)) <= 2e-3 * np.max(np.abs(lu_ref))


def test_partial_pivoting_reports_exact_singularity_and_solves(ctx):
    from grim_20261007_b200 import _lib
    from grim_20261007_b200.device import ptr
    a = _rand(150, 150, 9)
    a[:, 70] = 0.0
    _t, ipiv, info = _getrf(ctx, a, pivot=_lib.PIVOT_PARTIAL)
    lu_ref, piv_ref, info_ref = sla.lapack.zgetrf(a)
    assert info == info_ref == 71
    np.testing.assert_array_equal(ipiv.cpu().numpy(), piv_ref + 1)
    a = _rand(300, 300, 10)
    b = _rand(300, 40, 11)
    t, ipiv, info = _getrf(ctx, a, pivot=_lib.PIVOT_PARTIAL)
    bt = _dev(b)
    _lib.check(ctx.lib.grim_zgetrs(ctx.h, 300, 40, ptr(t), 300, ptr(ipiv), ptr(bt), 300))
    x_ref = np.linalg.solve(a, b)
    assert np.max(np.abs(_host(bt) - x_ref)) <= 1e-10 * np.max(np.abs(x_ref))


@pytest.mark.parametrize('n', [1, 7, 64, 97, 200, 333])
def test_zgetrf_matches_lapack_with_pivoting(ctx, n):
    a = _rand(n, n, n)
    t, ipiv, info = _getrf(ctx, a)
    lu_ref, piv_ref = sla.lu_factor(a)
    assert info == 0
    np.testing.assert_array_equal(ipiv.cpu().numpy(), piv_ref + 1)
    lu = _host(t)
    assert np.max(np.abs(lu - lu_ref)) <= 1e-11 * max(1.0, np.max(np.abs(lu_ref)))


@pytest.mark.parametrize('n', [64, 130, 256])
def test_zgetrf_diagonal_certificate_path(ctx, n):
    a = _rand(n, n, 100 + n, dominant=True)
    t, ipiv, info = _getrf(ctx, a)
    lu_ref, piv_ref = sla.lu_factor(a)
    assert np.all(piv_ref == np.arange(n))
    np.testing.assert_array_equal(ipiv.cpu().numpy(), np.arange(1, n + 1))
    assert ctx.lib.grim_launch_count(ctx.h) > 0
    from grim_20261007_b200 import _lib
    st = _lib.GrimSolveInfo()
    ctx.lib.grim_last_solve_info(ctx.h, ctypes.byref(st))
    assert st.pivoted_panels == 0
    assert np.max(np.abs(_host(t) - lu_ref)) <= 1e-12 * np.max(np.abs(lu_ref))


def test_zgetrf_reports_exact_singularity(ctx):
    a = _rand(70, 70, 3)
    a[:, 5] = 0.0
    _t, _ipiv, info = _getrf(ctx, a)
    lu_ref, piv_ref, info_ref = sla.lapack.zgetrf(a)
    assert info == info_ref == 6


@pytest.mark.parametrize('n,nrhs', [(97, 1), (200, 33), (256, 720)])
def test_zgetrs_multi_rhs(ctx, n, nrhs):
    from grim_20261007_b200 import _lib
    from grim_20261007_b200.device import ptr
    a = _rand(n, n, 7 * n)
    b = _rand(n, nrhs, 11 * n)
    t, ipiv, info = _getrf(ctx, a)
    bt = _dev(b)
    _lib.check(ctx.lib.grim_zgetrs(ctx.h, n, nrhs, ptr(t), n, ptr(ipiv), ptr(bt), n))
    x = _host(bt)
    x_ref = sla.lu_solve(sla.lu_factor(a), b)
    assert np.max(np.abs(x - x_ref)) <= 1e-10 * np.max(np.abs(x_ref))


def test_cgetrf_matches_lapack_complex64(ctx):
    n = 160
    a = _rand(n, n, 5).astype(np.complex64)
    t, ipiv, info = _getrf(ctx, a, complex64=True)
    lu_ref, piv_ref = sla.lu_factor(a)
    np.testing.assert_array_equal(ipiv.cpu().numpy(), piv_ref + 1)
    assert np.max(np.abs(_host(t) - lu_ref)) <= 2e-4 * np.max(np.abs(lu_ref))


def test_reference_dense_systems_at_the_gpu_hook(ctx):
    """B1 parity: the reference's own assembled systems, solved through grim_zgesv_batched."""
    from grim_20261007_b200.twod.solver import _solve_dense_gpu, _solve_dense_system
    d = np.load(os.path.join(GOLDEN, 'ref_dense_system.npz'))
    names = sorted({k[:-2] for k in d.files if k.endswith('_a')})
    assert len(names) >= 7
    for name in names:
        a, b, x_ref = d[name + '_a'], d[name + '_b'], d[name + '_x']
        x, dev = _solve_dense_gpu(a, b)
        assert isinstance(dev, str) and dev
        assert np.max(np.abs(x - x_ref)) <= 1e-10 * np.max(np.abs(x_ref)), name
        r = a @ x - b
        berr = np.max(np.abs(r), axis=0) / (np.max(np.sum(np.abs(a), axis=1)) * np.max(np.abs(x), axis=0)
                                            + np.max(np.abs(b), axis=0))
        assert np.max(berr) <= 1e-12, name
        x2 = _solve_dense_system(a, b, None, name)
        assert np.max(np.abs(x2 - x_ref)) <= 1e-10 * np.max(np.abs(x_ref))
    # the 2x2 system of the reference's own hook test: rtol 2e-14
    x, _ = _solve_dense_gpu(d['tiny_a'], d['tiny_b'][:, 0])
    np.testing.assert_allclose(d['tiny_a'] @ x, d['tiny_b'][:, 0], rtol=2e-14, atol=2e-14)


def test_mixed_solve_refines_to_fp64(ctx):
    from grim_20261007_b200.execution import linear_precision
    from grim_20261007_b200.twod.solver import _solve_dense_gpu
    d = np.load(os.path.join(GOLDEN, 'ref_dense_system.npz'))
    a, b, x_ref = d['cyl96_ka5_TM_a'], d['cyl96_ka5_TM_b'], d['cyl96_ka5_TM_x']
    with linear_precision('mixed'):
        x, _ = _solve_dense_gpu(a, b)
    assert np.max(np.abs(x - x_ref)) <= 1e-9 * np.max(np.abs(x_ref))
    rel = np.max(np.abs(a @ x - b), axis=0) / np.max(np.abs(b), axis=0)
    assert np.max(rel) <= 2e-12


def test_backward_error_kernel_matches_host(ctx):
    from grim_20261007_b200 import _lib
    from grim_20261007_b200.device import ptr
    n, m = 150, 9
    a = _rand(n, n, 1)
    x = _rand(n, m, 2)
    b = a @ x + 1e-6 * _rand(n, m, 3)
    at, xt, bt = _dev(a), _dev(x), _dev(b)
    berr = torch.empty(m, dtype=torch.float64, device='cuda')
    _lib.check(ctx.lib.grim_backward_error(ctx.h, n, m, ptr(at), n, 0, ptr(xt), n, ptr(bt), n, ptr(berr)))
    r = a @ x - b
    ref = np.max(np.abs(r), axis=0) / (np.max(np.sum(np.abs(a), axis=1)) * np.max(np.abs(x), axis=0)
                                       + np.max(np.abs(b), axis=0))
    np.testing.assert_allclose(berr.cpu().numpy(), ref, rtol=1e-6)


def test_mixed_falls_back_to_fp64_when_refinement_stalls(ctx):
    """complex64 LU of a kappa ~ 1e10 system cannot refine to 2e-12: the ladder solves it in FP64."""
    from grim_20261007_b200.execution import linear_precision
    from grim_20261007_b200.twod.solver import _solve_dense_gpu
    rng = np.random.default_rng(4)
    n = 96
    u, _ = np.linalg.qr(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    v, _ = np.linalg.qr(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    a = (u * np.logspace(0, -10, n)) @ v.conj().T
    b = rng.standard_normal((n, 3)) + 1j * rng.standard_normal((n, 3))
    with linear_precision('mixed'):
        x, _ = _solve_dense_gpu(a, b)
    r = a @ x - b
    berr = np.max(np.abs(r), axis=0) / (np.max(np.sum(np.abs(a), axis=1)) * np.max(np.abs(x), axis=0)
                                        + np.max(np.abs(b), axis=0))
    assert np.max(berr) < 1e-14


def test_backward_error_reports_nonfinite_solutions_as_infinite():
    """A NaN anywhere in a column's solution or residual makes that column's backward error
    infinite (a max that dropped NaN would report it as tiny)."""
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from grim_20261007_b200.device import to_device_colmajor
    from grim_20261007_b200.twod import operators as ops
    rng = np.random.default_rng(4)
    a = rng.standard_normal((80, 80)) + 1j * rng.standard_normal((80, 80))
    x = rng.standard_normal((80, 3)) + 0j
    b = a @ x
    x[5, 1] = np.nan
    berr = ops.backward_error(to_device_colmajor(a), to_device_colmajor(x), to_device_colmajor(b)).cpu().numpy()
    assert berr[0] < 1e-14 and berr[2] < 1e-14
    assert np.isinf(berr[1])


def _golden_matrices():
    import importlib.util
    path = os.path.join(GOLDEN, 'make_quality_gate_golden.py')
    spec = importlib.util.spec_from_file_location('make_quality_gate_golden', path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.matrices()


def test_condition_estimate_matches_the_exact_equilibrated_condition_and_the_reference(ctx):
    """grim_zcond1_equilibrated (Hager-Higham on the device) against the exact cond_1 of the
    row/column-equilibrated matrix and the reference's own estimate (SciPy's block estimator,
    tests/golden/quality_gate.json): a lower bound, within a factor 3 of both (equal to
    rounding on these matrices when the iteration finds the maximising column)."""
    import json
    from grim_20261007_b200.twod import operators as ops
    with open(os.path.join(GOLDEN, 'quality_gate.json')) as f:
        conds = json.load(f)['conditions']
    for a, ref in zip(_golden_matrices(), conds):
        est = ops.condition_estimate(_dev(a), ctx=ctx)
        assert est <= ref['exact'] * (1 + 1e-9), (a.shape, est, ref)
        assert est >= ref['exact'] / 3.0, (a.shape, est, ref)
        assert ref['reference_estimate'] / 3.0 <= est <= 3.0 * ref['reference_estimate']
    sing = _rand(50, 50, 77)
    sing[:, 20] = 0.0
    assert ops.condition_estimate(_dev(sing), ctx=ctx) == float('inf')
    assert ops.condition_estimate(_dev(np.array([[2.0 + 1.0j]])), ctx=ctx) == pytest.approx(1.0)


def _tournament_pivots(a, nb=64, rows=128):
    """NumPy model of the tournament (tslu.cuh): per panel, partial-pivoting selections on
    128-row blocks, then on the concatenated choices of sibling pairs up to the root (first
    row of the list on ties); the root's order is the panel's pivot order.  Returns the
    LAPACK-style ipiv (1-based) of the whole factorization."""
    a = np.array(a, dtype=np.complex128)
    n = a.shape[0]
    ipiv = np.zeros(n, dtype=np.int64)

    def select(rows_idx, panel, w):
        blk = panel[rows_idx].copy()
        alive = np.ones(len(rows_idx), bool)
        out = []
        for k in range(min(w, len(rows_idx))):
            v = np.where(alive, np.abs(blk[:, k].real) + np.abs(blk[:, k].imag), -1.0)
            p = int(np.argmax(v))
            out.append(rows_idx[p])
            alive[p] = False
            piv = blk[p, k]
            if piv != 0:
                l = np.where(alive, blk[:, k] / piv, 0)
                blk[:, k + 1:] -= np.outer(l, blk[p, k + 1:])
        return out

    for j in range(0, n, nb):
        w = min(nb, n - j)
        panel = a[j:, j:j + w]
        m = panel.shape[0]
        lists = [select(list(range(s, min(m, s + rows))), panel, w) for s in range(0, m, rows)]
        while len(lists) > 1:
            lists = [select(lists[i] + (lists[i + 1] if i + 1 < len(lists) else []), panel, w)
                     for i in range(0, len(lists), 2)]
        win = lists[0][:w]
        # swap sequence bringing win[s] to place s, applied to the whole matrix
        order = list(range(m))
        for s, r in enumerate(win):
            p = order.index(r)
            ipiv[j + s] = j + p + 1
            order[s], order[p] = order[p], order[s]
            a[[j + s, j + p]] = a[[j + p, j + s]]
        # eliminate the panel without pivoting, then the trailing update
        for k in range(w):
            a[j + k + 1:, j + k] /= a[j + k, j + k]
            a[j + k + 1:, j + k + 1:j + w] -= np.outer(a[j + k + 1:, j + k], a[j + k, j + k + 1:j + w])
        if j + w < n:
            l11 = np.tril(a[j:j + w, j:j + w], -1) + np.eye(w)
            a[j:j + w, j + w:] = sla.solve_triangular(l11, a[j:j + w, j + w:], lower=True, unit_diagonal=True)
            a[j + w:, j + w:] -= a[j + w:, j:j + w] @ a[j:j + w, j + w:]
    return ipiv, a


@pytest.mark.parametrize('n', [1, 5, 64, 130, 300, 1000, 2048, 2100, 4100])
def test_tournament_getrf_is_an_lu_with_the_tournament_pivots(ctx, n):
    """Tournament pivoting (tslu.cuh): P A = L U to FP64 accuracy, bounded multipliers, and
    the pivots of the NumPy model of the same tree (one CTA, 16 and 33 leaves; a last panel
    of 4 columns; 1 and 5 rows)."""
    from grim_20261007_b200 import _lib
    a = _rand(n, n, 900 + n)
    t, ipiv, info = _getrf(ctx, a, pivot=_lib.PIVOT_TOURNAMENT)
    assert info == 0
    piv = ipiv.cpu().numpy()
    assert np.all(piv >= np.arange(1, n + 1)) and np.all(piv <= n)
    lu = _host(t)
    low = np.tril(lu, -1) + np.eye(n)
    up = np.triu(lu)
    assert np.max(np.abs(low)) <= 10.0
    pa = a[_lapack_perm(piv)]
    assert np.max(np.abs(pa - low @ up)) <= 1e-11 * np.max(np.abs(a)) * max(1.0, n / 1000)
    if n <= 1000:
        ref_piv, ref_lu = _tournament_pivots(a)
        np.testing.assert_array_equal(piv, ref_piv)
        assert np.max(np.abs(lu - ref_lu)) <= 1e-10 * max(1.0, np.max(np.abs(ref_lu)))


@pytest.mark.parametrize('n', [300, 2048])
def test_tournament_cgetrf_and_mixed_solve(ctx, n):
    """complex64 tournament LU (the trailing update's packed operands written by the L21
    stage) is an LU of A to FP32 accuracy, and the mixed solve through it refines to FP64
    (backward error <= 1e-12 against LAPACK's solution)."""
    from grim_20261007_b200 import _lib
    from grim_20261007_b200.twod import operators as ops
    a = _rand(n, n, 77 + n)
    a32 = a.astype(np.complex64)
    t, ipiv, info = _getrf(ctx, a32, complex64=True, pivot=_lib.PIVOT_TOURNAMENT)
    assert info == 0
    lu = _host(t).astype(np.complex128)
    low = np.tril(lu, -1) + np.eye(n)
    up = np.triu(lu)
    pa = a32.astype(np.complex128)[_lapack_perm(ipiv.cpu().numpy())]
    assert np.max(np.abs(pa - low @ up)) <= 1e-4 * np.max(np.abs(a))
    rhs = _rand(n, 40, 5 + n)
    b = _dev(rhs)  # (40, n): the right-hand sides column-major
    st = ops.solve_inplace(_dev(a), b, 'mixed', tol=1e-13, stop='berr', pivot='tournament', tuned=False)
    xs = _host(b)
    ref = np.linalg.solve(a, rhs)
    assert np.max(np.abs(xs - ref)) <= 1e-9 * np.max(np.abs(ref))
    assert st['backward_error'] <= 1e-12


def test_tournament_singular_column_reports_info(ctx):
    from grim_20261007_b200 import _lib
    n = 300
    a = _rand(n, n, 12)
    a[:, 77] = 0.0
    _t, _ipiv, info = _getrf(ctx, a, pivot=_lib.PIVOT_TOURNAMENT)
    assert info == 78
