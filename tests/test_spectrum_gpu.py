"""GPU parity of the Radon spectrum, the guided picker and the SoftMax gradient against the oracle.

Tolerances: the GPU evaluates the DFT at the kept bins directly in FP64 while the
oracle uses an FFT, so spectra agree to ~1e-12 relative (1e-9 asserted).  Picks
are integer decisions on identical inputs and must match exactly.
"""
import numpy as np
import pytest

from swd_b200 import configs, spectrum as SP

pytestmark = pytest.mark.gpu


def _seis(O, s, is_=2):
    inp = O.fd_inputs(s.nbc, s.nt, s.dtx, s.dx, s.dt, int(s.sx[is_ - 1]), 1, s.gx, np.ones(s.ng), s.vp, s.vs,
                      in_wf=s.nt_wf)
    _, sw, _ = O.mex_staggerfd(inp, s.source())
    return sw.astype(np.float64)


def _rel(a, b):
    return np.linalg.norm(np.ravel(a - b)) / max(np.linalg.norm(np.ravel(b)), 1e-300)


@pytest.mark.parametrize("survey,shots", [("tiny", [1, 2, 3]), ("plain", [1, 6, 12])])
def test_radon_matches_oracle(O, survey, shots):
    s = configs.tiny(nt=400) if survey == "tiny" else configs.plain_c1()
    for is_ in shots:
        seis = _seis(O, s, is_)
        for side, fn in (("r", SP.RTrAD), ("l", SP.RTlAD)):
            ml, n, save = fn(seis, is_, s.df, s.dt, None, s.vmin, s.vmax, s.fmin, s.fmax, s.nt, s.ng, s.ds,
                             s.offset, s.m, s.M, s.dv)
            rml, rn, rsave = O.radon(seis, is_, s.df, s.dt, s.vmin, s.vmax, s.fmin, s.fmax, s.ng, s.ds, s.offset,
                                     s.m, s.M, side, s.dv)
            assert n == rn
            assert save["uxtposr" if side == "r" else "uxtposl"].tolist() == rsave["uxtpos"]
            assert _rel(ml, rml) < 1e-9
            assert _rel(save["mlr" if side == "r" else "mll"], rsave["ml_raw"]) < 1e-9
            assert _rel(save["mm"], rsave["mm"]) < 1e-9
            assert save["lf"] == rsave["lf"] and save["nf"] == rsave["nf"] and save["ccn"] == rsave["ccn"]


def test_radon_unit_velocity_step_is_reference_formula(O):
    """dv = 1 reproduces pp = 1./(vmin:vmax)' of RTrAD.m:20 exactly."""
    s = configs.tiny(nt=400)
    seis = _seis(O, s, 1)
    ml, n, save = SP.RTrAD(seis, 1, s.df, s.dt, 301, 100, 400, s.fmin, s.fmax, s.nt, s.ng, s.ds, s.offset, s.m, s.M)
    rml, _, _ = O.radon(seis, 1, s.df, s.dt, 100, 400, s.fmin, s.fmax, s.ng, s.ds, s.offset, s.m, s.M, "r", 1.0)
    assert ml.shape == (301, s.npair) and _rel(ml, rml) < 1e-9


def _random_spectra(rng, np_, npair, levels=None):
    ml = rng.random((np_, npair))
    if levels:  # quantise to force plateaus and ties
        ml = np.round(ml * levels) / levels + 1e-3
    # a drifting ridge so the walk has something to follow
    c = np.linspace(0.6, 0.3, npair) * np_
    p = np.arange(np_)[:, None]
    ml = ml * 0.4 + np.exp(-((p - c[None, :]) / (0.05 * np_)) ** 2)
    if levels:
        ml = np.round(ml * levels) / levels
    return ml / ml.max(0, keepdims=True)


@pytest.mark.parametrize("levels", [None, 8, 3])
@pytest.mark.parametrize("seed", range(6))
def test_pick_bit_exact_on_identical_spectra(O, levels, seed):
    rng = np.random.default_rng(seed)
    np_, npair = int(rng.integers(20, 400)), int(rng.integers(12, 80))
    ml = _random_spectra(rng, np_, npair, levels)
    cr0 = rng.integers(1, np_, npair).astype(float) + 100
    ini = int(rng.integers(1, npair + 1))
    try:
        rres, rcr = O.LHDispPick(ml, 100, cr0, 1, ini)
    except ValueError:
        with pytest.raises(Exception):
            SP.LHDispPick(ml, 100, cr0, 1, ini)
        return
    res, cr = SP.LHDispPick(ml, 100, cr0, 1, ini)
    assert np.array_equal(cr, rcr)
    assert res == pytest.approx(rres, rel=1e-12, abs=1e-12)


def test_pick_edges(O):
    """Walk hitting the last velocity (idx == a branch of pickFDC1.m:22), argmax ties, method 2."""
    np_, npair = 30, 15
    ml = np.full((np_, npair), 0.1)
    ml[-1, :6] = 1.0          # columns 1..6 peak at the last row
    ml[5, 6:] = 1.0
    ml[7, 6:] = 1.0           # tie: first index wins
    ml[2, :] = 0.05           # a local minimum
    cr0 = np.arange(npair) + 100.0
    for ini in (1, 3, 8, 15):
        rres, rcr = O.LHDispPick(ml, 100, cr0, 1, ini)
        res, cr = SP.LHDispPick(ml, 100, cr0, 1, ini)
        assert np.array_equal(cr, rcr), ini
    rres2, rcr2 = O.LHDispPick(ml, 100, cr0, 2, 1)
    res2, cr2 = SP.LHDispPick(ml, 100, cr0, 2, 1)
    assert np.array_equal(cr2, rcr2) and res2 == pytest.approx(rres2)


def test_pick_rejects_nan(O):
    ml = np.ones((10, 5))
    ml[3, 2] = np.nan
    with pytest.raises(Exception):
        SP.LHDispPick(ml, 100, np.zeros(5), 1, 2)


@pytest.mark.parametrize("survey,shots", [("tiny", [1, 2, 3]), ("plain", [1, 5, 12])])
def test_adwdgrad_matches_oracle(O, survey, shots):
    s = configs.tiny(nt=400) if survey == "tiny" else configs.plain_c1()
    rng = np.random.default_rng(7)
    for is_ in shots:
        seis = _seis(O, s, is_)
        saves = {}
        for side in ("r", "l"):
            saves[side] = O.radon(seis, is_, s.df, s.dt, s.vmin, s.vmax, s.fmin, s.fmax, s.ng, s.ds, s.offset, s.m,
                                  s.M, side, s.dv)[2]
        npair = saves["r"]["nf"] - saves["r"]["lf"] + 1
        gr = rng.integers(-3, 4, npair).astype(float)
        gl = rng.integers(-3, 4, npair).astype(float)
        ref = O.ADWDgrad_1(s.nt, s.ng, s.ns, npair, is_, s.w, s.m, s.M, s.soft_arg_norm, gr, gl, saves["r"],
                           saves["l"])
        p = SP.radon_params(s.df, s.dt, s.vmin, s.vmax, s.fmin, s.fmax, s.nt, s.ng, s.ds, s.offset, s.m, s.M, s.dv)
        gs = {k: {"mm": v["mm"], ("mlr" if k == "r" else "mll"): v["ml_raw"], "params": p} for k, v in saves.items()}
        got = SP.ADWDgrad_1(s.nt, s.ng, s.ns, npair, is_, s.w, s.m, s.M, s.soft_arg_norm, gr, gl, None, gs["r"],
                            gs["l"])
        assert np.abs(ref).max() > 0
        assert _rel(got, ref) < 1e-9, is_
        assert np.array_equal(np.abs(got).sum(0) > 0, np.abs(ref).sum(0) > 0)


@pytest.mark.parametrize("survey,shots", [("tiny", [1, 2, 3]), ("plain", [1, 6, 12])])
def test_adwdgrad_norm_matches_oracle(O, survey, shots):
    """ADWDgrad_norm: the SoftMax weights replaced by normpdf around the picks."""
    s = configs.tiny(nt=400) if survey == "tiny" else configs.plain_c1()
    rng = np.random.default_rng(8)
    for is_ in shots:
        seis = _seis(O, s, is_)
        saves = {}
        for side in ("r", "l"):
            saves[side] = O.radon(seis, is_, s.df, s.dt, s.vmin, s.vmax, s.fmin, s.fmax, s.ng, s.ds, s.offset, s.m,
                                  s.M, side, s.dv)[2]
        npair = saves["r"]["nf"] - saves["r"]["lf"] + 1
        npv = saves["r"]["ml_raw"].shape[0]
        gr = rng.integers(-3, 4, npair).astype(float)
        gl = rng.integers(-3, 4, npair).astype(float)
        cr_r = rng.integers(1, npv, npair).astype(float)
        cr_l = rng.integers(1, npv, npair).astype(float) + 0.5  # interpolated picks are not integers
        ref = O.ADWDgrad_norm(s.nt, s.ng, s.ns, npair, is_, s.w, s.m, s.M, s.soft_arg_norm, gr, gl, saves["r"],
                              saves["l"], cr_r, cr_l)
        p = SP.radon_params(s.df, s.dt, s.vmin, s.vmax, s.fmin, s.fmax, s.nt, s.ng, s.ds, s.offset, s.m, s.M, s.dv)
        gs = {"r": {"mm": saves["r"]["mm"], "mlr": saves["r"]["ml_raw"], "params": p, "cr_r": cr_r},
              "l": {"mm": saves["l"]["mm"], "mll": saves["l"]["ml_raw"], "params": p, "cr_l": cr_l}}
        got = SP.ADWDgrad_norm(s.nt, s.ng, s.ns, npair, is_, s.w, s.m, s.M, s.soft_arg_norm, gr, gl, None, gs["r"],
                               gs["l"])
        assert np.abs(ref).max() > 0
        assert _rel(got, ref) < 1e-9, is_


@pytest.mark.parametrize("beta", [1.0, 2.5])
def test_adwdgrad_limband_matches_oracle(O, beta):
    """ADWDgradlimband: power-normalised weights and the 25-bin ramps below lf and above nf.
    fmin 30 Hz puts lf at 31 (the ramp needs lf >= 26); SoftArgNorm stays small, since the
    reference's mlr.^SoftArgNorm overflows at SWD.m's 1e4."""
    import dataclasses
    s = dataclasses.replace(configs.plain_c1(), fmin=30.0)
    rng = np.random.default_rng(9)
    for is_ in (1, 6, 12):
        seis = _seis(O, s, is_)
        saves = {}
        for side in ("r", "l"):
            saves[side] = O.radon(seis, is_, s.df, s.dt, s.vmin, s.vmax, s.fmin, s.fmax, s.ng, s.ds, s.offset, s.m,
                                  s.M, side, s.dv)[2]
        npair = saves["r"]["nf"] - saves["r"]["lf"] + 1
        gr = rng.integers(-3, 4, npair).astype(float)
        gl = rng.integers(-3, 4, npair).astype(float)
        ref = O.ADWDgradlimband(s.nt, s.ng, s.ns, npair, is_, s.w, s.m, s.M, beta, gr, gl, saves["r"], saves["l"])
        p = SP.radon_params(s.df, s.dt, s.vmin, s.vmax, s.fmin, s.fmax, s.nt, s.ng, s.ds, s.offset, s.m, s.M, s.dv)
        gs = {k: {"mm": v["mm"], ("mlr" if k == "r" else "mll"): v["ml_raw"], "params": p} for k, v in saves.items()}
        got = SP.ADWDgradlimband(s.nt, s.ng, s.ns, npair, is_, s.w, s.m, s.M, beta, gr, gl, None, gs["r"], gs["l"])
        assert np.abs(ref).max() > 0
        assert _rel(got, ref) < 1e-9, is_

