"""CPU checks of the oracle itself (no GPU).

The reference ships no golden vectors, so the oracle is pinned here by
(1) two independent restatements of the FD loops agreeing bit for bit,
(2) closed-form properties of the setup functions, (3) documented behaviour of
MATLAB's findpeaks/interp1/max/round, and (4) physical known answers (a plane
wave's Radon peak sits at its phase velocity; the Radon pair is adjoint).
"""
import math

import numpy as np
import pytest

from swd_b200 import configs


def _tiny_inputs(O, single, src="w", nt=300, seed=0):
    rng = np.random.default_rng(seed)
    nz, nx, nbc = 7, 15, 5
    vs = 200 + 100 * rng.random((nz, nx))
    vp = 1.8 * vs
    dx, dt = 0.5, 1e-4
    inp = O.fd_inputs(nbc, nt, dt / dx, dx, dt, 6, 2, np.arange(1, nx + 1), np.ones(nx), vp, vs, source_type=src,
                      single=single)
    ainp = O.fd_inputs(nbc, nt, dt / dx, dx, dt, 6, 2, np.arange(1, nx + 1), np.ones(nx), vp, vs, single=single,
                       adjoint=True)
    s = configs.ricker(150.0, dt, nt)
    return inp, ainp, s, rng


@pytest.mark.parametrize("single", [True, False])
@pytest.mark.parametrize("src", ["w", "p", "s", "s1", "z"])
def test_fd_forward_two_restatements_agree(O, single, src):
    inp, _, s, _ = _tiny_inputs(O, single, src)
    su, sw, wf = O.mex_staggerfd(inp, s)
    su2, sw2, wf2 = O.fd_forward_np(inp, s.astype(inp.temp.dtype))
    assert np.abs(sw).max() > 0
    assert np.array_equal(sw, sw2) and np.array_equal(su, su2)
    for k in wf:
        assert np.array_equal(wf[k], wf2[k]), k


@pytest.mark.parametrize("single,acc64", [(True, True), (True, False), (False, True)])
def test_fd_adjoint_two_restatements_agree(O, single, acc64):
    inp, ainp, s, rng = _tiny_inputs(O, single)
    _, _, wf = O.mex_staggerfd(inp, s)
    res = rng.standard_normal((inp.iv[0].astype(int), 15)).astype(inp.temp.dtype)
    a = O.mex_e2drtm(ainp, res, wf, accum_fp64=acc64)
    b = O.fd_adjoint_np(ainp, res, wf, accum_fp64=acc64)
    for x, y in zip(a, b):
        assert np.abs(x).max() > 0
        assert np.array_equal(x, y)


def test_fd_single_close_to_double(O):
    inp32, _, s, _ = _tiny_inputs(O, True, nt=600)
    inp64, _, _, _ = _tiny_inputs(O, False, nt=600)
    _, sw32, _ = O.mex_staggerfd(inp32, s)
    _, sw64, _ = O.mex_staggerfd(inp64, s)
    rel = np.linalg.norm(sw32 - sw64) / np.linalg.norm(sw64)
    assert rel < 1e-4


def test_fd_adjoint_is_transpose_of_forward_on_receivers(O):
    """The reference adjoint is exact up to its material-in-derivative form: check <Fs, r> ~ <s, F^T r> loosely
    through energy: an impulse residual at a receiver produces a finite, decaying adjoint image."""
    inp, ainp, s, rng = _tiny_inputs(O, False, nt=300)
    _, _, wf = O.mex_staggerfd(inp, s)
    res = np.zeros((300, 15))
    res[150, 7] = 1.0
    cl, cm, il = O.mex_e2drtm(ainp, res, wf)
    assert np.all(np.isfinite(cl)) and np.abs(cl).max() > 0
    assert np.all(il >= 0)


def test_damp_circle_profile(O):
    nbc, nz, nx, top, dx, vmin = 6, 5, 9, 2, 0.5, 150.0
    d = O.damp_circle(vmin, nz + top + nbc, nx + 2 * nbc, nbc, dx, 1, top)
    a = (nbc - 1) * dx
    kappa = 3.0 * vmin * math.log(1e7) / (2.0 * a)
    assert d.shape == (nz + top + nbc, nx + 2 * nbc)
    assert np.all(d[top:top + nz, nbc:nbc + nx] == 0)          # interior undamped
    assert np.all(d[:top, :] == 0)                             # free surface: no top band or corners
    assert d[top, 0] == pytest.approx(kappa)                   # outermost left column = damp1d(nbc)
    assert d[-1, nbc] == pytest.approx(kappa)                  # bottom row
    assert np.allclose(d[:, :nbc], d[:, ::-1][:, :nbc])        # left/right symmetry
    dd = O.damp_circle(vmin, nz + 2 * nbc, nx + 2 * nbc, nbc, dx, 0, nbc)
    assert dd[0, 0] > 0 and np.allclose(dd, dd[::-1, :])       # no free surface: 4-fold symmetric


def test_ricker_peak_and_length():
    w = configs.ricker(30.0, 1e-4, 1000)
    nw = 2 * math.floor(2.2 / 30 / 1e-4 / 2) + 1
    assert np.argmax(w) == nw // 2 and w.max() == pytest.approx(1.0)
    assert np.all(w[nw:] == 0)


def test_pad_replicates_edges(O):
    p0 = np.arange(12.0).reshape(3, 4)
    p = O.pad(p0, 2, 1, 2)
    assert p.shape == (3 + 2 + 2, 4 + 4)
    assert np.all(p[:2, 2:6] == p0[0]) and np.all(p[-2:, 2:6] == p0[-1])
    assert np.all(p[2:5, 0] == p0[:, 0]) and p[0, 0] == p0[0, 0] and p[-1, -1] == p0[-1, -1]


@pytest.mark.parametrize("y,locs", [
    ([0, 1, 0], [2]),
    ([0, 1, 1, 0], [2]),                 # flat peak: first index
    ([0, 1, 1, 2, 0], [4]),              # rising plateau is not a peak
    ([1, 0, 1], []),                     # endpoints are never peaks
    ([0, 2, 1, 3, 1, 3], [2, 4]),
    ([3, 3, 3], []),
    ([0, 1, 1], []),                     # plateau running to the end
])
def test_findpeaks_semantics(O, y, locs):
    assert O.findpeaks_locs(np.asarray(y, float)) == locs


def test_mround_half_away_from_zero(O):
    assert [O.mround(v) for v in (0.5, 1.5, 2.5, -0.5, -2.5, 2.4999)] == [1, 2, 3, -1, -3, 2]


def test_interp_picks(O):
    idx = np.array([5, 7, 7, 9, 4, 4])
    ch = np.array([0, 1, 0, 1, 1, 0])
    out = O.interp_picks(idx, ch)
    assert out.tolist() == [7.0, 7.0, 8.0, 9.0, 4.0, 4.0]


def _ridge(np_, npair, center, width=3.0, seed=0):
    rng = np.random.default_rng(seed)
    p = np.arange(1, np_ + 1)[:, None]
    c = np.asarray(center, float)[None, :]
    ml = np.exp(-((p - c) / width) ** 2) + 0.01 * rng.random((np_, npair))
    return ml / ml.max(0, keepdims=True)


def test_pick_follows_single_ridge(O):
    np_, npair = 60, 20
    center = np.linspace(40, 20, npair)
    ml = _ridge(np_, npair, center)
    cr, dvmin, dvmax, idx, ch = O.pickFDC1(ml, 10, 2, 4)
    assert np.all(np.abs(idx - center) <= 1.5)
    res, cr_pre = O.LHDispPick(ml, 100, cr + 100, 1, 10)
    assert res == 0.0


def test_radon_plane_wave_peak(O):
    """A linear event moving at v0 gives its Radon maximum at p = 1/v0 at every frequency."""
    nt, ng, dt, dx = 1024, 40, 1e-3, 1.0
    v0 = 300.0
    t = np.arange(nt) * dt
    x = np.arange(ng) * dx
    w = configs.ricker(25.0, dt, nt)
    seis = np.zeros((nt, ng))
    for j in range(ng):
        shift = int(round(x[j] / v0 / dt))
        seis[shift:, j] = w[:nt - shift]
    ml, n, save = O.radon(seis, 1, 1.0, dt, 100, 600, 10, 40, ng, dx, 40, 0, 1, "r", dv=1.0)
    vel = O.velocities(100, 600, 1.0)
    peaks = vel[np.argmax(ml, axis=0)]
    assert np.all(np.abs(peaks - v0) < 15)


def test_radon_adjoint_dot_product(O):
    """<K d, g> == <d, K^H g> for the per-frequency Radon operator used by RTrAD/ADWDgrad_1."""
    rng = np.random.default_rng(0)
    pp = 1.0 / O.velocities(100, 400, 3.0)
    x = np.arange(20) * 0.5
    th = 2 * math.pi * 1.0 * np.outer(pp, x) * 17
    K = np.exp(1j * th)
    d = rng.standard_normal(20) + 1j * rng.standard_normal(20)
    g = rng.standard_normal(pp.size) + 1j * rng.standard_normal(pp.size)
    assert np.vdot(g, K @ d) == pytest.approx(np.vdot(K.conj().T @ g, d))


def test_smooth2a_box_mean(O):
    rng = np.random.default_rng(1)
    A = rng.standard_normal((7, 9))
    S = O.smooth2a(A, 1, 2)
    ref = np.zeros_like(A)
    for i in range(7):
        for j in range(9):
            ref[i, j] = A[max(0, i - 1):i + 2, max(0, j - 2):j + 3].mean()
    assert np.allclose(S, ref, rtol=1e-14, atol=1e-14)


def test_adwdgrad_sides_disjoint(O):
    """Right side writes the source trace and everything right of it; left writes strictly left of it."""
    s = configs.tiny(nt=400)
    seis = np.random.default_rng(0).standard_normal((s.nt, s.ng))
    is_ = 2
    _, _, sr = O.radon(seis, is_, s.df, s.dt, s.vmin, s.vmax, s.fmin, s.fmax, s.ng, s.ds, s.offset, s.m, s.M, "r",
                       s.dv)
    _, _, sl = O.radon(seis, is_, s.df, s.dt, s.vmin, s.vmax, s.fmin, s.fmax, s.ng, s.ds, s.offset, s.m, s.M, "l",
                       s.dv)
    npair = sr["nf"] - sr["lf"] + 1
    a = O.ADWDgrad_1(s.nt, s.ng, s.ns, npair, is_, s.w, s.m, s.M, s.soft_arg_norm, np.ones(npair), np.zeros(npair),
                     sr, sl)
    src_col = s.M * is_ - s.M + 1
    nz_cols = np.nonzero(np.abs(a).sum(0))[0] + 1
    assert nz_cols.min() >= max(1, src_col - s.offset) and nz_cols.max() <= min(s.ng, src_col + s.offset - 1)


def test_normpdf_weights_match_scipy(O):
    """paddingMl_norm.m's normpdf(1:np, cr, 16) against scipy's normal density."""
    from scipy.stats import norm
    cr = np.array([1.0, 17.5, 80.0, 140.0])
    w = O.normpdf_cols(141, cr)
    ref = norm.pdf(np.arange(1, 142)[:, None], loc=cr[None, :], scale=16.0)
    np.testing.assert_allclose(w, ref, rtol=1e-13, atol=0)


@pytest.mark.parametrize("F1", [0, 1])
def test_wd_restatement_matches_direct_low_bin_filter(O, F1):
    """weight_data_muti3 (FFT, bin loop, conjugate mirror) against the same filter written as
    x + (2/ntpad) Re sum_k (fac_k - 1) X_k e^{2 pi i k t/ntpad}: bin bookkeeping, window
    columns, offsets and the strict left-side rule."""
    rng = np.random.default_rng(11)
    nt, ng, dt, df, fmin, fmax = 300, 40, 1e-3, 2.0, 10.0, 40.0
    ntpad = int(1 / dt / df)
    ind = int(fmin / df + 1)
    npair = int((fmax - fmin) / df + 1)
    win = npair + 2 * ind
    offset, m, M, w, ns, dg = 12, 0, 3, 3, 12, 0.5
    refsx = np.floor((1 + 3 * np.arange(ns)) / 1) + 1
    obs, pred = rng.standard_normal((nt, ng)), rng.standard_normal((nt, ng))
    cr0, cr0l = 300 + 50 * rng.random(npair), 300 + 50 * rng.random(npair)
    crp, crpl = cr0 + rng.integers(-20, 21, npair), cr0l + rng.integers(-20, 21, npair)
    fre = 2 * np.pi * O.mlinspace(fmin, fmax, npair)
    for is_ in (1, 2, 5, 12):
        got = O.weight_data_muti3(obs, pred, is_, dt, df, offset, dg, F1, w, M, m, ns, refsx, win, fmin, fmax, cr0,
                                  cr0l, crp, crpl, ind)
        want = np.zeros((nt, ng))
        src = obs if F1 else pred
        rs = int(refsx[is_ - 1])
        sides = []
        if is_ <= ns - m // M - round(w / M):
            cols = np.arange(rs + m, min(m + offset - 1 + rs, ng) + 1)
            sides.append((cols, (m + np.arange(cols.size)) * dg, cr0, crp))
        if is_ > round(w / M) + m // M + 1:
            cols = np.arange(max(rs - offset - m, 0) + 1, rs - m + 1)
            sides.append((cols, (m + np.arange(cols.size)[::-1]) * dg, cr0l, crpl))
        for cols, y, c0, cp in sides:
            dk = np.zeros(win)
            dk[ind - 1:ind - 1 + npair] = fre * (c0 - cp) / (c0 * cp)
            for j, c in enumerate(cols):
                th = dk * y[j]
                fac = -1j * th / (2 * np.pi) * (np.exp(-1j * th) if F1 else 1)
                xp = np.zeros(ntpad)
                xp[:nt] = src[:, c - 1]
                want[:, c - 1] = O.wd_direct(xp, 1, fac, ntpad)[:nt]
        assert np.abs(want).max() > 0
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-12 * np.abs(want).max())
        if is_ == 1:  # no left side for the first shots
            assert not np.any(got[:, :rs - 1])
