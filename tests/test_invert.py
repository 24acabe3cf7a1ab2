"""The SWD inversion loop (swd_b200.invert): line-search rules on synthetic misfits (CPU) and
two iterations on the engine against the same loop driven by the oracle (GPU)."""
import dataclasses

import numpy as np
import pytest

from swd_b200 import configs
from swd_b200.invert import Inversion, clip, iterate, parabola_step


def test_parabola_step_finds_the_vertex():
    for fs, a, c in [(0.3, 2.0, 1.0), (1.7, 0.5, 3.0), (-0.2, 1.0, 0.1)]:
        res = lambda f: a * (f - fs) ** 2 + c  # noqa: E731
        for f1, f2 in [(0.5, 1.0), (0.25, 0.5), (0.125, 0.25)]:
            assert parabola_step(f1, f2, res(0.0), res(f1), res(f2)) == pytest.approx(fs, rel=1e-12, abs=1e-12)
    assert parabola_step(0.5, 1.0, 1.0, 1.0, 1.0) == 0.0 or np.isnan(parabola_step(0.5, 1.0, 1.0, 1.0, 1.0))


def test_clip_keeps_nan_and_bounds():
    v = clip(np.array([1.0, 5.0, np.nan, 12.0]), 2.0, 10.0)
    assert v[0] == 2.0 and v[1] == 5.0 and np.isnan(v[2]) and v[3] == 10.0


@pytest.mark.parametrize("fs", [0.9, 0.1, 0.02])
def test_iterate_on_a_quadratic_misfit(fs):
    """misfit quadratic in the step along dk: the search lands on its minimum, whichever branch
    (doubling to 2*f1, or halving f1 while the misfit rises) it takes."""
    rng = np.random.default_rng(0)
    vs = 300.0 + rng.random((6, 7))
    dk = rng.standard_normal((6, 7))
    pur = -0.05
    alpha = np.sqrt(np.sum(vs * vs)) / np.sqrt(np.sum(dk * dk)) * pur
    target = vs + alpha * fs * dk
    calls = []

    def misfit(v):
        calls.append(v)
        return float(np.mean((v - target) ** 2)) + 1.0

    vs1, _, info, f1 = iterate(vs, lambda v: (dk, misfit(v)), misfit, 0.0, 1e9, pur, 0.5)
    assert info["gama"] == pytest.approx(fs, rel=1e-9)
    np.testing.assert_allclose(vs1, target, rtol=1e-12)
    assert info["res0"] == pytest.approx(1.0, abs=1e-12)
    if fs > 0.25:
        assert info["f2"] == 1.0 and info["misfit_passes"] == 3
    else:
        assert info["f1"] < 0.5 and info["misfit_passes"] >= 3


@pytest.mark.gpu
def test_two_iterations_on_the_engine_match_the_oracle_loop(O):
    s = configs.tiny(nt=400, ns=5)
    vs0 = np.repeat(np.linspace(np.min(s.vs_true), np.max(s.vs_true), s.nz)[:, None], s.nx, 1)
    inv = Inversion(s, vs0, s.vs_true, err=0.01)
    hist = inv.run(2)
    vs_eng = inv.vs.copy()
    inv.close()
    # the same two iterations with the oracle's gradient and misfit
    vp = vs0 * s.vp_ratio
    vs, f1, offset = vs0.copy(), 0.5, s.offset
    vsmin, vsmax = float(np.min(s.vs_true)), float(np.max(s.vs_true))
    for k in (1, 2):
        so = dataclasses.replace(s, offset=offset)
        cr, cl = O.observed_curves(so, s.vs_true, vp=vp)

        def gradient(v):
            g = O.gradient(so, v, cr, cl, vp=vp)
            return g["dk_vs"], g["residual"]

        vs1, _, info, f1 = iterate(vs, gradient, lambda v: O.misfit(so, v, cr, cl, vp=vp), vsmin, vsmax, -0.05, f1)
        h = hist[k - 1]
        assert h.offset == offset
        assert h.residual == pytest.approx(info["residual"], rel=1e-12)
        for key in ("res1", "res2", "res3", "res0", "f1", "f2", "gama"):
            assert getattr(h, key) == pytest.approx(info[key], rel=1e-6, abs=1e-12), key
        assert h.alpha == pytest.approx(info["alpha"], rel=1e-5)
        if k > 1 and (info["residual"] - info["res0"]) / info["residual"] < 0.01:
            offset -= 3
            f1 = 0.5
        vs = vs1
    assert np.linalg.norm(vs_eng - vs) / np.linalg.norm(vs) < 1e-6
