"""The field-data variants (fieldexamples/outcrop, fieldexamples/QadimahFault) against the oracle.

* LHDispPick of the field drivers: the guided pick starts at the global maximum of the
  unnormalised spectrum (pickFDCValue seeded with its row, or pickFDC1 from its column) and the
  misfit leaves out the first and last rows (15..end-15, or 50..end-30).
* norm_trace: every predicted trace over its largest magnitude (0/0 = NaN for a dead trace).
* ADWDgrad_1 of the field drivers: the adjoint source over its largest magnitude.
* The shot loop of outcrop.m with manual-pick observed curves (the caller's curves).

Picks are integer decisions on identical inputs and match exactly; the misfit to 1e-12, the
adjoint source and the FP64 gradient to 1e-9 (the GPU's direct DFT against the oracle's FFT).
"""
import dataclasses

import numpy as np
import pytest

from swd_b200 import configs


def _ridge(rng, np_, npair, top=None):
    """A spectrum with a dispersive ridge plus noise, its unnormalised form and the column maxima
    placed so that the global maximum sits at column `top`."""
    p = np.arange(np_)[:, None]
    c = np.linspace(0.7, 0.3, npair) * np_
    raw = rng.random((np_, npair)) + 3.0 * np.exp(-0.5 * ((p - c[None, :]) / 5.0) ** 2)
    if top is not None:
        raw[:, top - 1] *= 1.5
    return raw / raw.max(axis=0, keepdims=True), raw


# ------------------------------------------------------------------ oracle (CPU)

def test_pickfdcvalue_is_pickfdc1_with_the_argmax_seed(O):
    rng = np.random.default_rng(1)
    ml, raw = _ridge(rng, 351, 56)
    for lp in (1, 10, 30, 56):
        a = O.pickFDC1(ml, lp, 2, 4)[0]
        b = O.pickFDCValue(ml, lp, int(np.argmax(ml[:, lp - 1])) + 1, 2, 4)[0]
        assert np.array_equal(a, b), lp


def test_field_misfit_leaves_out_the_edge_rows(O):
    rng = np.random.default_rng(2)
    ml, raw = _ridge(rng, 301, 120, top=40)
    _, cr = O.LHDispPick_field(ml, raw, 100, np.zeros(120), 1, 1)
    cr0 = cr.copy()
    cr0[:14] += 7.0   # rows 1..14 and 106..120 are outside 15..end-15
    cr0[-15:] -= 3.0
    assert O.LHDispPick_field(ml, raw, 100, cr0, 1, 1)[0] == 0.0
    cr0[14] += 2.0    # row 15 is inside
    assert O.LHDispPick_field(ml, raw, 100, cr0, 1, 1)[0] == pytest.approx(4.0 / (120 - 29))
    # variant 2: rows 50..end-30; an empty range gives NaN (mean([]))
    assert np.isnan(O.LHDispPick_field(ml[:, :60], raw[:, :60], 100, cr0[:60], 1, 2)[0])


def test_norm_trace_oracle(O):
    d = np.random.default_rng(3).standard_normal((50, 6))
    d[:, 2] = 0.0
    out = O.norm_trace(d)
    assert np.all(np.isnan(out[:, 2]))
    ok = [0, 1, 3, 4, 5]
    assert np.allclose(np.abs(out[:, ok]).max(0), 1.0)


def _fk_by_offset_operator(d):
    """The f-k filter as the GPU computes it: time DFT of the padded traces, one wavenumber
    operator per frequency half (h_plus for u_f < nf/2, h_minus otherwise), inverse time DFT."""
    ns, ntr = d.shape
    nf, nk = 2 * ns, 2 * ntr
    T = np.fft.fft(np.vstack([d, np.zeros_like(d)]), axis=0)  # nf x ntr
    u = np.arange(nk)
    m = (np.arange(ntr)[None, :] - np.arange(ntr)[:, None]) % nk  # [x, x'] -> x' - x mod nk
    e = np.exp(2j * np.pi * np.outer(np.arange(nk), u) / nk) / nk  # [m, u_k]
    hp, hm = e[:, u >= nk // 2].sum(1), e[:, u < nk // 2].sum(1)
    R = np.where((np.arange(nf) < nf // 2)[:, None], T @ hp[m], T @ hm[m])
    return np.real(np.fft.ifft(R, axis=0))[:ns]


def test_fk_filter_oracle_and_the_gpu_algebra(O):
    rng = np.random.default_rng(6)
    for ns, ntr in ((40, 7), (33, 1), (64, 12)):
        d = rng.standard_normal((ns, ntr))
        ref = O.fk_filter(d, 1e-3, 0.5)
        assert np.allclose(_fk_by_offset_operator(d), ref, rtol=0, atol=1e-12 * np.abs(ref).max())
    # a dip filter: an event whose arrival time grows with the trace index passes, the opposite
    # dip is mostly removed
    t, x = np.arange(128)[:, None], np.arange(16)[None, :]
    fwd = np.exp(-0.5 * ((t - 20 - 3.0 * x) / 2.0) ** 2)
    bwd = np.exp(-0.5 * ((t - 70 + 3.0 * x) / 2.0) ** 2)
    assert np.linalg.norm(O.fk_filter(fwd, 1e-3, 0.5)) > 0.8 * np.linalg.norm(fwd)
    assert np.linalg.norm(O.fk_filter(bwd, 1e-3, 0.5)) < 0.3 * np.linalg.norm(bwd)


# ------------------------------------------------------------------ GPU

@pytest.mark.gpu
@pytest.mark.parametrize("variant,method", [(1, 1), (1, 2), (2, 1)])
def test_field_picker_matches_oracle(O, variant, method):
    from swd_b200 import spectrum as SP
    rng = np.random.default_rng(10 + variant)
    for top, npair in ((40, 120), (1, 100), (100, 100)):
        ml, raw = _ridge(rng, 351, npair, top=top)
        cr0 = rng.integers(100, 400, npair).astype(float)
        ref = O.LHDispPick_field(ml, raw, 100, cr0, method, variant)
        got = SP.LHDispPick_field(ml, 100, cr0, method, {"mlr": raw, "uxtposr": np.arange(5.0)}, variant)
        assert np.array_equal(got[1], ref[1]), (top, npair)
        assert got[0] == pytest.approx(ref[0], rel=1e-12)
        # the left side's state carries mll instead
        got_l = SP.LHDispPick_field(ml, 100, cr0, method, {"mll": raw, "uxtposl": np.arange(5.0)}, variant)
        assert np.array_equal(got_l[1], ref[1])


@pytest.mark.gpu
def test_norm_trace_matches_oracle(O):
    from swd_b200 import spectrum as SP
    d = np.random.default_rng(4).standard_normal((777, 33)) * 1e-3
    d[:, 5] = 0.0
    d[100, 7] = np.nan  # MATLAB's max skips NaN; the NaN sample stays NaN
    ref = O.norm_trace(d)
    got = SP.norm_trace(d)
    assert np.array_equal(got, ref, equal_nan=True)


@pytest.mark.gpu
def test_maxnorm_adjoint_source_matches_oracle(O):
    from swd_b200 import spectrum as SP
    s = configs.plain_c1()
    rng = np.random.default_rng(9)
    for is_ in (1, 6, 12):
        inp = O.fd_inputs(s.nbc, s.nt, s.dtx, s.dx, s.dt, int(s.sx[is_ - 1]), 1, s.gx, np.ones(s.ng), s.vp, s.vs,
                          in_wf=s.nt_wf)
        seis = O.mex_staggerfd(inp, s.source())[1].astype(np.float64)
        saves = {side: O.radon(seis, is_, s.df, s.dt, s.vmin, s.vmax, s.fmin, s.fmax, s.ng, s.ds, s.offset, s.m,
                               s.M, side, s.dv)[2] for side in ("r", "l")}
        npair = saves["r"]["nf"] - saves["r"]["lf"] + 1
        gr = rng.integers(-3, 4, npair).astype(float)
        gl = rng.integers(-3, 4, npair).astype(float)
        args = (s.nt, s.ng, s.ns, npair, is_, s.w, s.m, s.M, s.soft_arg_norm, gr, gl)
        ref = O.ADWDgrad_1_maxnorm(*args, saves["r"], saves["l"])
        p = SP.radon_params(s.df, s.dt, s.vmin, s.vmax, s.fmin, s.fmax, s.nt, s.ng, s.ds, s.offset, s.m, s.M, s.dv)
        gs = {k: {"mm": v["mm"], ("mlr" if k == "r" else "mll"): v["ml_raw"], "params": p} for k, v in saves.items()}
        got = SP.ADWDgrad_1_maxnorm(*args, None, gs["r"], gs["l"])
        assert np.nanmax(np.abs(got)) == 1.0
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-9, is_


@pytest.mark.gpu
@pytest.mark.parametrize("field,FK", [(1, 0), (2, 0), (2, 1)])
def test_field_shot_loop_with_manual_picks_matches_oracle(O, field, FK):
    """outcrop.m's shot loop in double (its wrappers call the _double MEX) with manual-pick
    observed curves: picks identical, gradient and misfit to 1e-9; FK=1 is QademahSWD3.m's
    f-k filter option (:119)."""
    from swd_b200 import swd_loop
    s = dataclasses.replace(configs.tiny(nt=400, ns=5), df=1.0)  # 161 frequencies: room for the edge rows
    cr0_r, cr0_l = O.observed_curves(s, s.vs_true, single=False)
    rng = np.random.default_rng(5)
    man_r = cr0_r + rng.integers(-4, 5, cr0_r.shape)  # "manual" picks: the true curves, hand-nudged
    man_l = cr0_l + rng.integers(-4, 5, cr0_l.shape)
    ref = O.gradient(s, s.vs, man_r, man_l, single=False, field=field, FK=FK)
    got = swd_loop.gradient(s, s.vs, man_r, man_l, single=False, field=field, FK=FK)
    assert np.array_equal(got["cr_pre_r"], ref["cr_pre_r"]) and np.array_equal(got["cr_pre_l"], ref["cr_pre_l"])
    for k in ("g_cl", "g_cm", "g_illum", "dk_vs"):
        assert np.linalg.norm(got[k] - ref[k]) / np.linalg.norm(ref[k]) < 1e-9, k
    np.testing.assert_allclose(got["res_r"], ref["res_r"], rtol=1e-12, equal_nan=True)


@pytest.mark.gpu
def test_fk_filter_matches_oracle(O):
    from swd_b200 import spectrum as SP
    rng = np.random.default_rng(7)
    for ns, ntr in ((400, 17), (37, 5), (1000, 1), (8000, 45)):  # 2*37: a 2 x 37 four-step split
        d = rng.standard_normal((ns, ntr))
        ref = O.fk_filter(d, 5e-5, 0.5)
        got = SP.fk_filter(d, 5e-5, 0.5)
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-12, (ns, ntr)


@pytest.mark.gpu
@pytest.mark.parametrize("side", ["r", "l"])
def test_radon_with_fk_filter_matches_oracle(O, side):
    """RTrAD/RTlAD with FK=1 (the field drivers' option): the gather, in the transform's trace
    order, is f-k filtered before the transform."""
    from swd_b200 import spectrum as SP
    s = configs.plain_c1()
    inp = O.fd_inputs(s.nbc, s.nt, s.dtx, s.dx, s.dt, int(s.sx[5]), 1, s.gx, np.ones(s.ng), s.vp, s.vs,
                      in_wf=s.nt_wf)
    seis = O.mex_staggerfd(inp, s.source())[1].astype(np.float64)
    for is_ in (1, 6, 12):
        ml_ref, n_ref, save_ref = O.radon(seis, is_, s.df, s.dt, s.vmin, s.vmax, s.fmin, s.fmax, s.ng, s.ds,
                                          s.offset, s.m, s.M, side, s.dv, FK=1)
        f = SP.RTrAD if side == "r" else SP.RTlAD
        ml, n, save = f(seis, is_, s.df, s.dt, None, s.vmin, s.vmax, s.fmin, s.fmax, s.nt, s.ng, s.ds, s.offset,
                        s.m, s.M, s.dv, FK=1)
        assert n == n_ref
        assert np.linalg.norm(ml - ml_ref) / np.linalg.norm(ml_ref) < 1e-9, is_
        assert np.linalg.norm(save["mm"] - save_ref["mm"]) / np.linalg.norm(save_ref["mm"]) < 1e-9, is_
        plain = f(seis, is_, s.df, s.dt, None, s.vmin, s.vmax, s.fmin, s.fmax, s.nt, s.ng, s.ds, s.offset, s.m,
                  s.M, s.dv)[0]
        if n > 2:  # a one-trace gather's normalised spectrum is all ones, filtered or not
            assert not np.allclose(plain, ml)  # the filter changed the spectrum


@pytest.mark.gpu
def test_qadimahfault_fd_wrappers_are_core_with_a_time_interval():
    """QademahSWD3.m's staggerfd_eigen / e2drtm_eigen take an unused fsz and the snapshot interval
    as a time (dt_wf = 10 dt there, :96): the same bits as core's wrappers with in_wf = 10."""
    from swd_b200 import fd as F
    s = configs.tiny(nt=400)
    w = s.source().astype(np.float32)
    geo = (1, s.nbc, s.nt, s.dtx, s.dx, s.dt, 5, 1, s.gx, np.ones(s.ng), w, s.vp, s.vs)
    su, sw, www = F.staggerfd_eigen(*geo, 1, 22, "w", 0, 10)
    fu, fw, fww = F.staggerfd_eigen_field(*geo, 1, 0, 22, "w", 0, 10 * s.dt, (s.nt - 1) // 10 + 1)
    assert np.array_equal(su, fu) and np.array_equal(sw, fw)
    for k in ("fux", "fuz", "bwx", "bwz"):
        assert np.array_equal(www[k], fww[k]), k
    res = np.asfortranarray(sw * 0.5)
    adj = (1, s.nbc, s.nt, s.dtx, s.dx, s.dt, s.gx, np.ones(s.ng), w, s.vp, s.vs)
    core = F.e2drtm_eigen(www, res, *adj, 1, 22, 0, 10)
    field = F.e2drtm_eigen_field(fww, res, *adj, 1, 0, 22, 0, 10 * s.dt)
    for a, b in zip(core, field):
        assert np.array_equal(a, b)
