"""The WD adjoint source weight_data_muti3 (core/weight_data_muti3.m) through the C ABI.

CPU tests check the argument rules (they fail before any device work); GPU tests compare
the CUDA filter with the oracle's FFT restatement on the same inputs.
"""
import numpy as np
import pytest

from swd_b200 import configs


def _case(rng, nt=300, ng=40, dt=1e-3, df=2.0, fmin=10.0, fmax=40.0, ns=12):
    ind = int(fmin / df + 1)
    npair = int((fmax - fmin) / df + 1)
    c = dict(nt=nt, ng=ng, dt=dt, df=df, fmin=fmin, fmax=fmax, ind=ind, npair=npair, win=npair + 2 * ind,
             offset=12, m=0, M=3, w=3, ns=ns, dg=0.5, refsx=np.floor((1 + 3 * np.arange(ns)) / 1) + 1)
    c["obs"], c["pred"] = rng.standard_normal((nt, ng)), rng.standard_normal((nt, ng))
    c["cr0"], c["cr0l"] = 300 + 50 * rng.random(npair), 300 + 50 * rng.random(npair)
    c["crp"] = c["cr0"] + rng.integers(-20, 21, npair)
    c["crpl"] = c["cr0l"] + rng.integers(-20, 21, npair)
    return c


def _call(f, c, is_, F1, **kw):
    c = dict(c, **kw)
    return f(c["obs"], c["pred"], is_, c["dt"], c["df"], c["offset"], c["dg"], F1, c["w"], c["M"], c["m"], c["ns"],
             c["refsx"], c["win"], c["fmin"], c["fmax"], c["cr0"], c["cr0l"], c["crp"], c["crpl"], c["ind"])


def _rel(a, b):
    return np.linalg.norm(np.ravel(a - b)) / np.linalg.norm(np.ravel(b))


@pytest.mark.parametrize("bad,match", [(dict(nt=600), "ntpad"), (dict(win=260), "2\\*win"),
                                       (dict(ind=30), "ind"), (dict(F1=2), "F1")])
def test_wd_rejects_cases_the_reference_bin_loop_does_not_handle(bad, match):
    from swd_b200 import spectrum as SP
    from swd_b200._lib import SwdError
    rng = np.random.default_rng(0)
    nt = bad.pop("nt", 300)
    c = _case(rng, nt=nt)
    F1 = bad.pop("F1", 0)
    with pytest.raises(SwdError, match=match):
        _call(SP.weight_data_muti3, c, 3, F1, **bad)


def test_wd_rejects_empty_window():
    from swd_b200 import spectrum as SP
    from swd_b200._lib import SwdError
    c = _case(np.random.default_rng(0))
    c["refsx"] = c["refsx"].copy()
    c["refsx"][4] = c["ng"] + 1  # right window starts past the last receiver
    with pytest.raises(SwdError, match="window"):
        _call(SP.weight_data_muti3, c, 5, 0)


@pytest.mark.gpu
@pytest.mark.parametrize("F1", [0, 1])
def test_wd_matches_oracle(O, F1):
    from swd_b200 import spectrum as SP
    c = _case(np.random.default_rng(5))
    for is_ in (1, 2, 3, 7, 11, 12):
        ref = _call(O.weight_data_muti3, c, is_, F1)
        got = _call(SP.weight_data_muti3, c, is_, F1)
        assert np.abs(ref).max() > 0
        assert _rel(got, ref) < 1e-12, is_
        assert np.array_equal(got != 0, ref != 0), is_


@pytest.mark.gpu
def test_wd_on_a_modelled_gather(O):
    """The plain 30x120 survey's predicted data (FP32 FD), SWD.m's ind/win and picks."""
    from swd_b200 import spectrum as SP
    s = configs.plain_c1()
    rng = np.random.default_rng(2)
    ind = s.fmin / s.df + 1
    win = s.npair + 2 * ind
    dgc = int(s.gx[1] - s.gx[0])
    refsx = np.floor(s.sx / dgc) + 1
    for is_ in (1, 6, 12):
        inp = O.fd_inputs(s.nbc, s.nt, s.dtx, s.dx, s.dt, int(s.sx[is_ - 1]), 1, s.gx, np.ones(s.ng), s.vp, s.vs,
                          source_type="w", in_wf=s.nt_wf)
        _, sw, _ = O.mex_staggerfd(inp, s.source(), want_wf=False)
        seis = sw.astype(np.float64)
        cr0 = 250 + 100 * rng.random(s.npair)
        crp = cr0 + rng.integers(-30, 31, s.npair)
        args = (None, seis, is_, s.dt, s.df, s.offset, s.ds, 0, s.w, s.M, s.m, s.ns, refsx, win, s.fmin, s.fmax,
                cr0, cr0[::-1], crp, crp[::-1], ind)
        ref = O.weight_data_muti3(seis, *args[1:])
        got = SP.weight_data_muti3(*args)
        assert _rel(got, ref) < 1e-12, is_


def test_adwdgrad_limband_rejects_low_lf():
    """The reference's ramp indexes column lf-25: with lf below 26 it fails, and so does the call
    (before any device work)."""
    from swd_b200 import spectrum as SP
    from swd_b200._lib import SwdError
    s = configs.plain_c1()  # fmin 5 Hz: lf = 6
    p = SP.radon_params(s.df, s.dt, s.vmin, s.vmax, s.fmin, s.fmax, s.nt, s.ng, s.ds, s.offset, s.m, s.M, s.dv)
    npv, npair = s.np_vel, s.npair
    gs = {"mm": np.zeros((npv, 61), complex), "mlr": np.ones((npv, npair)), "params": p}
    with pytest.raises(SwdError, match="lf - 25"):
        SP.ADWDgradlimband(s.nt, s.ng, s.ns, npair, 2, s.w, s.m, s.M, 1.0, np.ones(npair), np.ones(npair), None,
                           gs, dict(gs, mll=gs["mlr"]))
