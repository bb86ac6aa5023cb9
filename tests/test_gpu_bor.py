"""GPU body-of-revolution path against the FP64 oracle, the reference solver and Mie."""
import os

import numpy as np
import pytest

from oracle import bor as OB, mie
from grim_20261007_b200 import synthetic as S
from tests.conftest import GOLDEN

pytestmark = pytest.mark.gpu
torch = pytest.importorskip('torch')


@pytest.fixture(scope='module')
def ctx():
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from grim_20261007_b200.device import context
    return context()


@pytest.mark.parametrize('alpha', [1.0, 0.5, 0.0])
@pytest.mark.parametrize('m', [0, 1, -1, 2, -3])
def test_mode_matrix_matches_oracle(ctx, m, alpha):
    """EFIE (alpha 1), CFIE (0.5) and MFIE (0) reduced matrices on a 14-element sphere."""
    from grim_20261007_b200.bor import solver as B
    pts = S.sphere_generatrix(1.0, 14)
    k, mmax = 2.5, 4
    dev = B.BorDevice(pts, k, mmax, alpha=alpha)
    Zg = dev.matrix(m).cpu().numpy().T
    body = OB.Body(pts)
    asm = OB.Assembler(body, k, mmax, mfie=alpha < 1.0)
    Q = OB.pole_transform(body, m)
    Zf = asm.matrix(m) if alpha == 1.0 else alpha * asm.matrix(m) + (1 - alpha) * OB.ETA0 * asm.mfie_matrix(m)
    Zr = Q.conj().T @ Zf @ Q
    assert np.max(np.abs(Zg - Zr)) <= 1e-11 * np.max(np.abs(Zr))


@pytest.mark.parametrize('name', ['sphere', 'graded'])
def test_mode_operators_match_reference(ctx, name):
    """The GPU's reduced EFIE / CFIE / MFIE matrices against the reference's own per-mode
    operators (tests/golden/ref_bor_modes.npz: its assemble_mode, assemble_mfie_mode)."""
    from grim_20261007_b200.bor import solver as B
    g = np.load(os.path.join(GOLDEN, 'ref_bor_modes.npz'))
    pts, k, mmax = g[f'{name}_points'], float(g[f'{name}_k']), int(g[f'{name}_mmax'])
    body = OB.Body(pts)
    for alpha in (1.0, 0.5, 0.0):
        dev = B.BorDevice(pts, k, mmax, alpha=alpha)
        for m in g['modes']:
            m = int(m)
            Q = OB.pole_transform(body, m)
            Zf = alpha * g[f'{name}_efie_{m}'] + (1 - alpha) * OB.ETA0 * g[f'{name}_mfie_{m}']
            Zr = Q.conj().T @ Zf @ Q
            Zg = dev.matrix(m).cpu().numpy().T
            assert np.max(np.abs(Zg - Zr)) <= 1e-11 * np.max(np.abs(Zr)), (alpha, m)


@pytest.mark.parametrize('alpha', [1.0, 0.5])
def test_excitation_matches_oracle(ctx, alpha):
    from grim_20261007_b200.bor import solver as B
    pts = S.ogive_generatrix(3.0, 22.0, 16)
    k = 4.0
    dev = B.BorDevice(pts, k, 3, alpha=alpha)
    th = torch.as_tensor(np.array([5.0, 47.0, 90.0, 133.0]), device='cuda')
    body = OB.Body(pts)
    for m in (-2, -1, 0, 1, 3):
        Q = OB.pole_transform(body, m)
        for far in (False, True):
            got = dev.excitation(m, th, far).cpu().numpy().T
            full = OB.excitation(body, k, th.cpu().numpy(), m, far=far)
            if not far and alpha < 1.0:
                full = alpha * full + (1 - alpha) * OB.excitation(body, k, th.cpu().numpy(), m, kind='mfie')
            ref = (Q.T if far else Q.conj().T) @ full
            assert np.max(np.abs(got - ref)) <= 1e-12 * max(1e-30, np.max(np.abs(ref)))


def test_solve_matches_oracle_and_mie(ctx):
    from grim_20261007_b200.bor.solver import solve_bor
    pts = S.sphere_generatrix(1.0, 24)
    k = 2.0
    th = [0.0, 35.0, 90.0, 160.0]
    res = solve_bor(pts, k * S.C0 / (2 * np.pi), th, formulation='efie', n_modes=6)
    o = OB.solve(pts, k, th, 6)
    for key in ('amp_vv', 'amp_hh'):
        got = np.asarray(res[key])
        assert np.max(np.abs(got - o[key])) <= 1e-9 * np.max(np.abs(o[key]))
    db = 10 * np.log10(np.asarray(res['sigma_vv']) / mie.sphere_sigma(1.0, k))
    assert np.max(np.abs(db)) < 0.1  # 24 elements: second-order discretisation error ~0.07 dB


def test_reference_sphere_golden(ctx):
    """Reference solve_bor (EFIE) on the 45-element sphere at ka = 3 (tests/golden/ref_bor_sphere.npz)."""
    from grim_20261007_b200.bor.solver import solve_bor
    g = np.load(os.path.join(GOLDEN, 'ref_bor_sphere.npz'))
    res = solve_bor(g['points'], float(g['freq_hz']), g['thetas'], formulation='efie', n_modes=int(g['modes_used']))
    for pol in ('vv', 'hh'):
        amp = np.asarray(res['amp_' + pol])
        ref = g['amp_%s_efie' % pol]
        assert np.max(np.abs(amp - ref)) <= 1e-8 * np.max(np.abs(ref))
    assert np.max(np.abs(10 * np.log10(np.asarray(res['sigma_vv']) / float(g['mie_sigma'])))) < 0.02
    assert res['n_unknowns'] == int(g['n_unknowns']) and res['formulation'] == 'efie'


def test_reference_cfie_default(ctx):
    """formulation='auto' on a closed body is the reference's CFIE: its far field of the
    45-element sphere at ka = 3 with its adaptive mode count (ref_bor_modes.npz)."""
    from grim_20261007_b200.bor.solver import solve_bor
    g = np.load(os.path.join(GOLDEN, 'ref_bor_modes.npz'))
    res = solve_bor(g['sphere45_points'], float(g['sphere45_freq_hz']), g['sphere45_thetas'])
    assert res['formulation'] == 'cfie' and res['modes_used'] == int(g['sphere45_modes_used'])
    for pol in ('vv', 'hh'):
        ref = g[f'sphere45_amp_{pol}']
        assert np.max(np.abs(np.asarray(res['amp_' + pol]) - ref)) <= 1e-8 * np.max(np.abs(ref))


def test_interior_resonance_cfie(ctx):
    """Next to the sphere's first interior resonance (ka = 2.7437) the EFIE and the CFIE
    each equal the reference's solve; the CFIE stays on Mie."""
    from grim_20261007_b200.bor.solver import solve_bor
    g = np.load(os.path.join(GOLDEN, 'ref_bor_modes.npz'))
    for form in ('efie', 'cfie'):
        res = solve_bor(g['resonant_points'], float(g['resonant_freq_hz']), g['resonant_thetas'], formulation=form,
                        n_modes=12)
        for pol in ('vv', 'hh'):
            ref = g[f'resonant_{form}_amp_{pol}']
            assert np.max(np.abs(np.asarray(res['amp_' + pol]) - ref)) <= 1e-7 * np.max(np.abs(ref)), (form, pol)
        if form == 'cfie':
            db = 10 * np.log10(res['sigma_vv'][0] / float(g['resonant_mie_sigma']))
            assert abs(db) < 0.05


@pytest.mark.parametrize('form', ['cfie', 'mfie'])
def test_cfie_and_mfie_solves_match_oracle(ctx, form):
    """solve_bor with formulation 'cfie' / 'mfie' against the oracle's solve of the same
    body (a 20-element ogive, |m| <= 5)."""
    from grim_20261007_b200.bor.solver import solve_bor
    pts = S.ogive_generatrix(3.0, 22.0, 20)
    k = 3.0
    th = [0.0, 40.0, 90.0, 155.0]
    res = solve_bor(pts, k * S.C0 / (2 * np.pi), th, formulation=form, n_modes=5)
    o = OB.solve(pts, k, th, 5, formulation=form)
    assert res['formulation'] == form
    for key in ('amp_vv', 'amp_hh'):
        got = np.asarray(res[key])
        assert np.max(np.abs(got - o[key])) <= 1e-9 * np.max(np.abs(o[key])), key


@pytest.mark.parametrize('m', [0, 1, -2])
def test_mirror_halves_solve_equals_full_lu(ctx, m):
    """Even / odd halves of a symmetric body's CFIE mode matrix: split, two half solves and
    the join equal the LU solve of the full matrix; the asymmetry check reads rounding."""
    from grim_20261007_b200.bor import solver as B
    from grim_20261007_b200.device import ptr
    pts = S.ogive_generatrix(3.0, 22.0, 30)
    dev = B.BorDevice(pts, 5.0, 4, alpha=0.5)
    th = torch.as_tensor(np.array([10.0, 60.0, 120.0]), device='cuda')
    Z = dev.matrix(m)
    V = dev.excitation(m, th, far=False)
    mp = dev.mirror(m)
    assert mp is not None
    n, nrhs = int(Z.shape[0]), int(V.shape[0])
    out = torch.empty(2, dtype=torch.float64, device='cuda')
    ctx.lib.grim_bor_mirror_asymmetry(ctx.h, n, ptr(Z), n, ptr(mp['target']), ptr(mp['sign']), ptr(out))
    d, a = out.cpu().numpy()
    assert d <= 1e-13 * a
    ref = np.linalg.solve(Z.cpu().numpy().T, V.cpu().numpy().T)
    outs = B._solve_mirror_grouped(dev, [m], [Z.clone()], [V], workers=1)
    assert outs[0]['mirror_halves'] == [mp['k'] + mp['nfe'], mp['k'] + mp['nfo']]
    got = V.cpu().numpy().T
    assert np.max(np.abs(got - ref)) <= 1e-11 * np.max(np.abs(ref))


def test_cfie_rejects_open_shells(ctx):
    from grim_20261007_b200.bor.solver import solve_bor
    pts = S.sphere_generatrix(1.0, 12)[:-2]  # ends off the axis
    with pytest.raises(ValueError):
        solve_bor(pts, 3e8, [0.0], formulation='cfie', n_modes=2)
    res = solve_bor(pts, 3e8, [0.0, 90.0], n_modes=2)
    assert res['formulation'] == 'efie'


def test_signed_mode_symmetry_matches_all_modes():
    """Solving m = 0..M with m > 0 counted twice equals summing every signed mode."""
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from grim_20261007_b200.bor.solver import solve_bor_device
    gen, _length, _half = S.ogive_case(6, n=40)
    k = 8.0 / float(np.max(gen[:, 0]))
    th = np.arange(0.0, 180.5, 7.5)
    f_half, t_half = solve_bor_device(gen, k, th, 9)
    f_all, t_all = solve_bor_device(gen, k, th, 9, signed_mode_symmetry=False)
    assert t_half['mode_systems_solved'] == 10 and t_all['mode_systems_solved'] == 19
    np.testing.assert_allclose(f_half, f_all, rtol=1e-11, atol=1e-11 * np.max(np.abs(f_all)))


@pytest.mark.parametrize('precision', ['double', 'mixed'])
def test_grouped_modes_match_per_mode_solves(precision, monkeypatch):
    """The mode systems factored by one grouped LU give the same far field as each mode
    factored on its own (identical factors, or on this mirror-symmetric ogive the even/odd
    halves; the mixed refinement stops at the same backward-error target).  Mixed: every
    mode is forced onto the complex64 path, whatever its order."""
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from grim_20261007_b200.bor import solver as bs
    from grim_20261007_b200.bor.solver import solve_bor_device
    monkeypatch.setattr(bs, 'MIXED_MIN_ORDER', 0)
    monkeypatch.setattr(bs, 'MIXED_MODE_FRACTION', 1e9)
    gen, _length, _half = S.ogive_case(8, n=60)
    k = 10.0 / float(np.max(gen[:, 0]))
    th = np.arange(0.0, 180.5, 5.0)
    f_g, t_g = solve_bor_device(gen, k, th, 12, precision=precision)
    f_1, t_1 = solve_bor_device(gen, k, th, 12, precision=precision, grouped=False)
    assert t_g['mode_systems_solved'] == t_1['mode_systems_solved'] == 13
    # double: the grouped path solves the symmetric ogive's modes through their mirror halves
    rtol = 1e-11 if precision == 'double' else 1e-8
    np.testing.assert_allclose(f_g, f_1, rtol=rtol, atol=rtol * np.max(np.abs(f_1)))
    # the release gate measured every mode against its full matrix
    limit = bs.release_limit(precision, 1e-10)
    for t in (t_g, t_1):
        assert 0.0 < t['max_backward_error'] <= limit
        assert 0.0 < t['max_relative_residual'] <= bs.BOR_LINEAR_RESIDUAL_MAX


def test_adaptive_mode_tail_matches_reference(ctx):
    """With the default mode cap the modal sum stops where the reference's adaptive tail
    stopped on the same sphere (tests/golden/ref_bor_sphere.npz: |m| <= 10)."""
    from grim_20261007_b200.bor.solver import solve_bor
    g = np.load(os.path.join(GOLDEN, 'ref_bor_sphere.npz'))
    res = solve_bor(g['points'], float(g['freq_hz']), g['thetas'], formulation='efie')
    assert res['modes_used'] == int(g['modes_used']) and res['mode_converged']
    assert res['mode_cap'] > res['modes_used']
    for pol in ('vv', 'hh'):
        amp = np.asarray(res['amp_' + pol])
        assert np.max(np.abs(amp - g['amp_%s_efie' % pol]) / np.abs(g['amp_%s_efie' % pol])) < 2e-3


@pytest.mark.parametrize('slices', [0, 8])
def test_solution_errors_match_numpy(ctx, slices):
    """grim_solution_errors: R = B - A X, the normwise backward error and the 2-norm
    relative residual per column (a zero right-hand side included) against NumPy."""
    from grim_20261007_b200.device import ptr
    rng = np.random.default_rng(17)
    n, nrhs = 300, 37
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    X = rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs))
    Bm = A @ X + 1e-9 * (rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs)))
    Bm[:, 5] = 0.0
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a.T), device='cuda')  # column-major storage
    Ad, Xd, Bd = dev(A), dev(X), dev(Bm)
    R = torch.empty_like(Bd)
    berr = torch.empty(nrhs, dtype=torch.float64, device='cuda')
    relres = torch.empty_like(berr)
    maxes = torch.empty(2, dtype=torch.float64, device='cuda')
    assert ctx.lib.grim_solution_errors(ctx.h, n, nrhs, ptr(Ad), n, ptr(Xd), n, ptr(Bd), n, ptr(R), n, slices,
                                        ptr(berr), ptr(relres), ptr(maxes)) == 0
    assert ctx.lib.grim_synchronize(ctx.h) == 0
    Rn = Bm - A @ X
    scale = np.max(np.abs(A)) * np.max(np.abs(X)) * n
    assert np.max(np.abs(R.cpu().numpy().T - Rn)) <= 1e-15 * scale
    anorm = np.max(np.sum(np.abs(A), axis=1))
    be = np.max(np.abs(Rn), axis=0) / (anorm * np.max(np.abs(X), axis=0) + np.max(np.abs(Bm), axis=0))
    bn = np.linalg.norm(Bm, axis=0)
    rr = np.linalg.norm(Rn, axis=0) / np.where(bn > 0, bn, 1.0)
    np.testing.assert_allclose(berr.cpu().numpy(), be, rtol=1e-4)
    np.testing.assert_allclose(relres.cpu().numpy(), rr, rtol=1e-4)
    np.testing.assert_allclose(maxes.cpu().numpy(), [be.max(), rr.max()], rtol=1e-4)


def _gate_case():
    from grim_20261007_b200.bor import solver as B
    pts = S.sphere_generatrix(1.0, 14)
    dev = B.BorDevice(pts, 2.5, 4, alpha=0.5)
    th = torch.as_tensor(np.arange(0.0, 181.0, 10.0), device='cuda')
    modes = [0, 1, 2]
    Zs = [dev.matrix(m) for m in modes]
    B0s = [dev.excitation(m, th, far=False) for m in modes]
    exact = [np.linalg.solve(Z.cpu().numpy().T, b.cpu().numpy().T) for Z, b in zip(Zs, B0s)]
    return B, modes, Zs, B0s, exact


def test_release_gate_refines_and_falls_back(ctx):
    """The per-mode release gate: a direct FP64 solution off by 1e-7 is refined from where it
    stands, a mirror / mixed one off by as much is replaced by the LU solution, an exact
    one is released untouched; every mode ends at the reference's limits."""
    B, modes, Zs, B0s, exact = _gate_case()
    rng = np.random.default_rng(3)
    Xs = []
    for i, x in enumerate(exact):
        # per-column noise: a column whose right-hand side vanishes (no excitation of this mode
        # at that aspect) keeps its exact zero solution, the only one with a small backward error
        noise = 1e-7 * np.max(np.abs(x), axis=0) * (rng.standard_normal(x.shape) + 1j * rng.standard_normal(x.shape))
        Xs.append(torch.as_tensor(np.ascontiguousarray((x + (noise if i < 2 else 0.0)).T), device='cuda'))
    out = B._gate_modes(modes, Zs, Xs, B0s, ['double', 'double', 'double'], [True, False, True], 1e-10)
    assert out[0]['gate_refinement_steps'] >= 1 and 'gate_lu_fallback' not in out[0]
    assert 'gate_lu_fallback' in out[1]
    assert out[2]['gate_refinement_steps'] == 0 and 'gate_lu_fallback' not in out[2]
    for o, X, x in zip(out, Xs, exact):
        assert o['backward_error'] <= B.BOR_LINEAR_BACKWARD_ERROR_MAX
        assert o['relative_residual'] <= B.BOR_LINEAR_RESIDUAL_MAX
        assert np.max(np.abs(X.cpu().numpy().T - x)) <= 1e-10 * np.max(np.abs(x))
    # a mixed solution is released at its refinement target, not at the FP64 limit
    x = exact[0]
    noise = 1e-13 * np.max(np.abs(x), axis=0) * (rng.standard_normal(x.shape) + 1j * rng.standard_normal(x.shape))
    Xm = torch.as_tensor(np.ascontiguousarray((x + noise).T), device='cuda')
    om = B._gate_modes([0], [Zs[0]], [Xm], [B0s[0]], ['mixed'], [False], 1e-10)[0]
    assert 'gate_lu_fallback' not in om and om['gate_refinement_steps'] == 0


def test_release_gate_raises_above_the_limit(ctx, monkeypatch):
    """A backward error that refinement cannot bring under the limit raises (the limit is
    set to zero here, so no solution can reach it)."""
    B, modes, Zs, B0s, exact = _gate_case()
    monkeypatch.setattr(B, 'BOR_LINEAR_BACKWARD_ERROR_MAX', 0.0)
    X = torch.as_tensor(np.ascontiguousarray(exact[0].T), device='cuda')
    with pytest.raises(RuntimeError, match='exceeds the release limit'):
        B._gate_modes([0], [Zs[0]], [X], [B0s[0]], ['double'], [True], 1e-10)


def _plain_factor(lu):
    """A scipy LU (logical (i, j) indexing) as the device factor entry of condition_estimates."""
    dt = torch.complex64 if lu.dtype == np.complex64 else torch.complex128
    t = torch.as_tensor(np.ascontiguousarray(lu.T), dtype=dt, device='cuda')
    return {'halves': None, 'lu': [t], 'ipiv': [None]}


def test_condition_estimates_match_lapack_zgecon(ctx):
    """grim_zcond1_factored on LAPACK's own LU factors equals 1 / zgecon (the reference's
    per-mode estimate) on random systems of ragged orders, all in one launch; complex64
    factors against cgecon to single precision."""
    import scipy.linalg as sl
    from scipy.linalg import lapack
    from grim_20261007_b200.bor import solver as B
    rng = np.random.default_rng(11)
    orders = [1, 2, 5, 31, 32, 33, 100, 257]
    mats, facs, ref = [], [], []
    for n in orders:
        A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)) + 3.0 * np.eye(n) * (n % 3 == 0)
        lu, _piv = sl.lu_factor(A)
        anorm = float(np.max(np.sum(np.abs(A), axis=0)))
        rcond, info = lapack.zgecon(lu, anorm, norm='1')
        assert info == 0
        mats.append(torch.as_tensor(np.ascontiguousarray(A.T), device='cuda'))
        facs.append(_plain_factor(lu))
        ref.append(1.0 / rcond)
    got = B.condition_estimates(mats, facs)
    np.testing.assert_allclose(got, ref, rtol=1e-9)
    # complex64 factors (the mixed path) against cgecon
    A = rng.standard_normal((120, 120)) + 1j * rng.standard_normal((120, 120))
    lu32, _piv = sl.lu_factor(A.astype(np.complex64))
    anorm = float(np.max(np.sum(np.abs(A), axis=0)))
    rc32, _info = lapack.cgecon(lu32, anorm, norm='1')
    got32 = B.condition_estimates([torch.as_tensor(np.ascontiguousarray(A.T), device='cuda')], [_plain_factor(lu32)])
    np.testing.assert_allclose(got32, [1.0 / rc32], rtol=1e-4)


def test_condition_estimates_of_mirror_halves_and_modes(ctx):
    """A mirror-split ogive mode: the estimate through its halves' LUs is a lower bound of the
    exact 1-norm condition number within a factor 3, as zgecon's on the full LU; the grouped
    mode solve reports the same estimates for its modes."""
    from grim_20261007_b200.bor import solver as B
    pts = S.ogive_generatrix(3.0, 22.0, 30)
    dev = B.BorDevice(pts, 5.0, 4, alpha=0.5)
    th = torch.as_tensor(np.array([10.0, 60.0, 120.0]), device='cuda')
    modes = [0, 1, 2, 3]
    Zs = [dev.matrix(m) for m in modes]
    Vs = [dev.excitation(m, th, far=False) for m in modes]
    outs, facs = B._solve_mirror_grouped(dev, modes, [z.clone() for z in Zs], Vs, workers=1, keep_factors=True)
    got = B.condition_estimates(Zs, facs)
    for Z, c in zip(Zs, got):
        z = Z.cpu().numpy().T
        exact = np.linalg.norm(z, 1) * np.linalg.norm(np.linalg.inv(z), 1)
        assert exact / 3.0 <= c <= exact * (1 + 1e-9), (c, exact)
    gen, _l, _h = S.ogive_case(8, n=60)
    k = 10.0 / float(np.max(gen[:, 0]))
    _f, tele = B.solve_bor_device(gen, k, np.arange(0.0, 180.5, 5.0), 6, alpha=0.5)
    assert tele['condition_est_computed'] and 1.0 < tele['median_cond'] <= tele['max_cond'] < B.BOR_CONDITION_EST_MAX
    _f1, tele1 = B.solve_bor_device(gen, k, np.arange(0.0, 180.5, 5.0), 6, alpha=0.5, grouped=False)
    # mirror halves (grouped) and full LUs (per mode) estimate the same condition numbers
    assert tele1['max_cond'] / 3.0 <= tele['max_cond'] <= 3.0 * tele1['max_cond']


def test_condition_gate_raises_above_the_limit(monkeypatch):
    """The reference's condition release limit: a mode estimated above it raises (the limit is
    lowered to 1 here, below every condition number)."""
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from grim_20261007_b200.bor import solver as B
    monkeypatch.setattr(B, 'BOR_CONDITION_EST_MAX', 1.0)
    pts = S.sphere_generatrix(1.0, 14)
    for grouped in (True, False):
        with pytest.raises(RuntimeError, match='condition .* exceeds the release limit'):
            B.solve_bor_device(pts, 2.5, [0.0, 45.0, 90.0], 3, alpha=0.5, grouped=grouped)


def test_release_gate_paths_when_every_mode_misses_the_limits(monkeypatch):
    """With the relative-residual limit at zero every mode misses the release limits: the
    grouped path replaces each mirror-halves solution by its full LU solution (and takes
    its condition estimate again), the per-mode path solves each mode again from its FP64
    LU; both far fields equal the ordinary solve's."""
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from grim_20261007_b200.bor import solver as B
    gen, _l, _h = S.ogive_case(5, n=40)
    k = 8.0 / float(np.max(gen[:, 0]))
    th = np.arange(0.0, 180.5, 15.0)
    f0, t0 = B.solve_bor_device(gen, k, th, 6, alpha=0.5)
    monkeypatch.setattr(B, 'BOR_LINEAR_RESIDUAL_MAX', 0.0)
    f1, t1 = B.solve_bor_device(gen, k, th, 6, alpha=0.5)
    assert len(t1.get('gate_lu_fallback_modes', [])) >= 1  # the mirror-split modes of this symmetric body
    f2, _t2 = B.solve_bor_device(gen, k, th, 6, alpha=0.5, grouped=False)
    for f in (f1, f2):
        np.testing.assert_allclose(f, f0, rtol=1e-10, atol=1e-10 * np.max(np.abs(f0)))
    assert t1['max_cond'] / 3.0 <= t0['max_cond'] <= 3.0 * t1['max_cond']
