"""Grouped LU of many systems of different orders (grim_getrf_grouped) against the
single-system factorization and LAPACK, and the grouped sweep solve against per-system
solves."""
import ctypes

import numpy as np
import pytest
import scipy.linalg as sla

pytestmark = pytest.mark.gpu

torch = pytest.importorskip('torch')

# orders: one panel, exact multiples of 64, ragged last panels, a long tail of small systems
ORDERS = [700, 64, 1, 513, 130, 257, 65, 1031, 200, 7, 384]


@pytest.fixture(scope='module')
def ctx():
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from grim_20261007_b200.device import context
    return context()


def _systems(seed):
    """Random complex systems; every third needs row interchanges (no diagonal boost)."""
    rng = np.random.default_rng(seed)
    out = []
    for i, n in enumerate(ORDERS):
        a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        if i % 3:
            a += np.diag(np.full(n, 4.0 * n))
        out.append(a)
    return out


def _single(ctx, a, dtype):
    from grim_20261007_b200 import _lib
    from grim_20261007_b200.device import ptr, to_device_colmajor
    n = a.shape[0]
    t = to_device_colmajor(a, dtype)
    ipiv = torch.zeros(n, dtype=torch.int32, device='cuda')
    info = ctypes.c_int(-1)
    fn = ctx.lib.grim_cgetrf if dtype == torch.complex64 else ctx.lib.grim_zgetrf
    _lib.check(fn(ctx.h, n, ptr(t), n, ptr(ipiv), ctypes.byref(info)))
    return t, ipiv, info.value


@pytest.mark.parametrize('dtype', ['complex128', 'complex64'])
@pytest.mark.parametrize('use_graph', [False, True])
def test_grouped_getrf_equals_single_and_lapack(ctx, dtype, use_graph):
    from grim_20261007_b200.device import to_device_colmajor, to_host_matrix
    from grim_20261007_b200.grouped import getrf_grouped
    dt = getattr(torch, dtype)
    mats = _systems(5)
    dev = [to_device_colmajor(a, dt) for a in mats]
    ipivs, infos, piv = getrf_grouped(dev, use_graph=use_graph, ctx=ctx)
    assert infos == [0] * len(mats)
    assert any(p > 0 for p in piv), 'the unboosted systems must exercise the pivoted fallback'
    for a, t, ip, npv in zip(mats, dev, ipivs, piv):
        n = a.shape[0]
        ts, ips, info = _single(ctx, a, dt)
        assert info == 0
        # same kernels per element, same fallback decisions: identical factors and pivots
        np.testing.assert_array_equal(ip.cpu().numpy(), ips.cpu().numpy())
        lu, lus = to_host_matrix(t), to_host_matrix(ts)
        assert np.array_equal(lu, lus), f'n={n}: max |grouped - single| {np.max(np.abs(lu - lus)):.3g}'
        if dtype == 'complex128':
            lu_ref, piv_ref = sla.lu_factor(a)
            np.testing.assert_array_equal(ip.cpu().numpy(), piv_ref + 1)
            assert np.max(np.abs(lu - lu_ref)) <= 1e-10 * np.max(np.abs(lu_ref))
        # P L U reconstructs A in any case
        L = np.tril(lu, -1) + np.eye(n)
        U = np.triu(lu)
        pa = a.astype(np.complex64).astype(complex) if dtype == 'complex64' else a.copy()
        for k, pk in enumerate(ip.cpu().numpy() - 1):
            pa[[k, pk]] = pa[[pk, k]]
        tol = 1e-4 if dtype == 'complex64' else 1e-12
        assert np.max(np.abs(L @ U - pa)) <= tol * np.max(np.abs(pa)) * max(1, n) ** 0.5


def test_grouped_graph_replay_on_new_matrices(ctx):
    """A second call with the same orders replays the captured graph on new matrices."""
    from grim_20261007_b200.device import to_device_colmajor, to_host_matrix
    from grim_20261007_b200.grouped import getrf_grouped
    first = [to_device_colmajor(a, torch.complex64) for a in _systems(11)]
    getrf_grouped(first, use_graph=True, ctx=ctx)
    l0 = ctx.lib.grim_launch_count(ctx.h)
    mats = _systems(12)
    dev = [to_device_colmajor(a, torch.complex64) for a in mats]
    ipivs, infos, _ = getrf_grouped(dev, use_graph=True, ctx=ctx)
    launched = ctx.lib.grim_launch_count(ctx.h) - l0
    assert infos == [0] * len(mats) and launched > 0
    for a, t, ip in zip(mats, dev, ipivs):
        ts, ips, _ = _single(ctx, a, torch.complex64)
        np.testing.assert_array_equal(ip.cpu().numpy(), ips.cpu().numpy())
        assert np.array_equal(to_host_matrix(t), to_host_matrix(ts))


def test_grouped_singular_system_reports_info(ctx):
    from grim_20261007_b200.device import to_device_colmajor
    from grim_20261007_b200.grouped import getrf_grouped
    rng = np.random.default_rng(3)
    good = rng.standard_normal((90, 90)) + 4 * 90 * np.eye(90)
    bad = rng.standard_normal((70, 70)) + 0j
    bad[:, 40] = 0.0  # column 40 zero: U(40, 40) == 0 under any row order
    dev = [to_device_colmajor(a, torch.complex128) for a in (good, bad)]
    _, infos, _ = getrf_grouped(dev, use_graph=False, ctx=ctx)
    assert infos[0] == 0 and infos[1] == 41


def test_grouped_sweep_matches_per_system_solves():
    """Mixed sweep through the grouped LU equals per-system mixed solves (both refined to a
    backward error of 1e-10 against the same complex64 matrices) and stays within 0.05 dB of
    FP64."""
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from grim_20261007_b200 import synthetic as S
    from grim_20261007_b200.twod import geometry as geo, operators as ops
    cases, _ = S.airfoil_sweep_case(1, nfreq=12, nmin=64, nmax=900)
    ang = np.arange(0.0, 180.0, 2.0)
    bodies = [ops.DeviceBody(geo.panel_geometry([v]), None) for v, _k, _f in cases]
    ks = [k for _v, k, _f in cases]
    for pol in ('TM', 'TE'):
        if pol == 'TE':
            bodies = [ops.DeviceBody(geo.panel_geometry([v]), geo.te_curvature_correction([v])) for v, _k, _f in cases]
        grouped = ops.monostatic_solves_grouped(bodies, ks, ang, pol, precision='mixed')
        for body, k, g in zip(bodies, ks, grouped):
            one = ops.monostatic_solve(body, k, ang, pol, precision='mixed')
            ref = ops.monostatic_solve(body, k, ang, pol, precision='double')
            a_g, a_1 = g['amplitude'].cpu().numpy(), one['amplitude'].cpu().numpy()
            a_64 = ref['amplitude'].cpu().numpy()
            assert g['telemetry']['backward_error'] <= 1e-10
            assert np.max(np.abs(a_g - a_1)) <= 1e-7 * np.max(np.abs(a_1))
            s64 = np.abs(a_64) ** 2
            db = 10 * np.log10(s64)
            mask = db > db.max() - 40
            assert np.max(np.abs(10 * np.log10(np.abs(a_g) ** 2 / s64))[mask]) < 0.05


@pytest.mark.parametrize('orders', [[1], [300], [1, 2, 3, 64, 65]])
def test_grouped_edge_orders(ctx, orders):
    """One system, 1 x 1 systems and orders around one panel: equal to the single-system LU."""
    from grim_20261007_b200.device import to_device_colmajor, to_host_matrix
    from grim_20261007_b200.grouped import getrf_grouped
    rng = np.random.default_rng(len(orders) * 7 + orders[0])
    mats = [rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)) + (2.0 * n if i % 2 else 0.0) * np.eye(n)
            for i, n in enumerate(orders)]
    for dt in (torch.complex64, torch.complex128):
        dev = [to_device_colmajor(a, dt) for a in mats]
        ipivs, infos, _ = getrf_grouped(dev, use_graph=True, ctx=ctx)
        assert infos == [0] * len(mats)
        for a, t, ip in zip(mats, dev, ipivs):
            ts, ips, info = _single(ctx, a, dt)
            assert info == 0
            np.testing.assert_array_equal(ip.cpu().numpy(), ips.cpu().numpy())
            assert np.array_equal(to_host_matrix(t), to_host_matrix(ts))
