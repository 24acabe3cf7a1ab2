"""The SWD inversion loop (SWD.m:143-337) on the batched engine.

Each iteration:

1. picks the observed dispersion curves at the current offset window (SWD.m:150-162);
2. runs one gradient pass, which gives residual(k) and the smoothed Vs gradient dk_vs
   (SWD.m:171-201);
3. sets the step scale alpha = ||vs|| / ||dk_vs|| * pur (SWD.m:206-209);
4. runs SWD.m's parabolic line search (SWD.m:210-306): misfit passes at f1 and 2*f1, or
   halving f1 while the misfit rises, the parabola's minimum gama, and the fallback to the
   better trial step when the parabola step is worse;
5. clips the new model to [vsmin, vsmax] (SWD.m:211, 308);
6. shrinks the offset window by 3 traces when the relative decrease of the misfit drops
   below `err`, resetting f1, and stops when the window reaches 3 traces (SWD.m:327-337).

As in SWD.m, vp stays that of the starting model, and the observed data are modelled with
that vp and the true Vs (SWD.m:138-140).  The loop logic is written once over two
callables, so the same iteration can run on the engine (`Inversion`) or on any other
implementation of the gradient and misfit passes.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Callable

import numpy as np


def clip(vs, vsmin, vsmax):
    """vs1(vs1<vsmin)=vsmin; vs1(vs1>vsmax)=vsmax (NaN is left as it is)."""
    v = np.array(vs, np.float64, copy=True)
    v[v < vsmin] = vsmin
    v[v > vsmax] = vsmax
    return v


def parabola_step(f1, f2, res0, res1, res2):
    """gama of SWD.m:285: the minimum of the parabola through (0,res0), (f1,res1), (f2,res2);
    an infinite value becomes 0 (SWD.m:287-289)."""
    num = f1 * f1 * (res0 - res2) + f2 * f2 * (res1 - res0)
    den = 2 * res0 * (f1 - f2) + 2 * res1 * f2 - 2 * res2 * f1
    with np.errstate(divide="ignore", invalid="ignore"):
        g = np.float64(num) / np.float64(den)
    return 0.0 if np.isinf(g) else float(g)


@dataclasses.dataclass
class Step:
    """What one iteration did (the values SWD.m prints)."""
    k: int
    offset: int
    residual: float       # residual(k): misfit of the model the gradient was taken at
    alpha: float
    f1: float
    f2: float
    res1: float
    res2: float
    gama: float
    res3: float
    res0: float           # misfit of the accepted model
    misfit_passes: int
    offset_next: int


def iterate(vs, gradient: Callable, misfit: Callable, vsmin, vsmax, pur=-0.05, f1=0.5):
    """One SWD iteration after the observed curves are set: gradient(vs) -> (dk_vs, residual),
    misfit(vs) -> residual.  Returns (new vs, Step fields, f1 to carry)."""
    dk, residual = gradient(vs)
    res0 = residual
    v_mean = math.sqrt(float(np.sum(vs * vs)))
    g_mean = math.sqrt(float(np.sum(dk * dk)))
    alpha = v_mean / g_mean * pur
    passes = 0

    def trial(f):
        nonlocal passes
        passes += 1
        return misfit(clip(vs + alpha * f * dk, vsmin, vsmax))

    res1 = trial(f1)
    f2, res2 = f1, res1
    if res1 > res0:
        while res1 > res0 and f1 > 0.0001:  # SWD.m:232-257
            f2, res2 = f1, res1
            f1 = f1 * 0.5
            res1 = trial(f1)
    else:  # SWD.m:258-283
        f2 = f1 * 2
        res2 = trial(f2)
    gama = parabola_step(f1, f2, res0, res1, res2)
    vs1 = clip(vs + alpha * gama * dk, vsmin, vsmax)
    res3 = misfit(vs1)
    passes += 1
    if res3 > res1 or res3 > res2:  # SWD.m:310-322
        if res1 > res2:
            res0, gama = res2, f2
        else:
            res0, gama = res1, f1
        vs1 = clip(vs + alpha * gama * dk, vsmin, vsmax)
    else:
        res0 = res3
    info = dict(residual=residual, alpha=alpha, f1=f1, f2=f2, res1=res1, res2=res2, gama=gama, res3=res3,
                res0=res0, misfit_passes=passes)
    return vs1, dk, info, f1


class Inversion:
    """SWD.m's inversion on the batched engine.

    survey: a configs.Survey (geometry, Radon and SoftMax settings, the starting offset);
    vs0: starting model; vs_true: the model that generates the observed data.
    """

    def __init__(self, survey, vs0, vs_true, vsmin=None, vsmax=None, pur=-0.05, err=0.01, offmin=3,
                 **engine_opts):
        self.survey = survey
        self.vs = np.asarray(vs0, np.float64).copy()
        self.vp = self.vs * survey.vp_ratio  # fixed: vp of the starting model (SWD.m:35)
        self.vs_true = np.asarray(vs_true, np.float64)
        self.vsmin = float(np.min(vs_true)) if vsmin is None else float(vsmin)
        self.vsmax = float(np.max(vs_true)) if vsmax is None else float(vsmax)
        self.pur, self.err, self.offmin = pur, err, offmin
        self.offset = int(survey.offset)
        self.f1 = 0.5
        self.k = 1
        self.history: list[Step] = []
        self._opts = engine_opts
        self._eng = None
        self._eng_offset = None

    def _engine(self):
        from .engine import GradientEngine
        if self._eng is None or self._eng_offset != self.offset:
            if self._eng is not None:
                self._eng.close()
            s = dataclasses.replace(self.survey, offset=self.offset)
            self._eng = GradientEngine(s, **self._opts)
            self._eng_offset = self.offset
            # observed curves at this window: the true model with the starting vp (SWD.m:138-162)
            cr, cl = self._eng.observed_curves(self.vp, self.vs_true)
            self._eng.set_observed(cr, cl)
        return self._eng

    def step(self):
        e = self._engine()

        def gradient(vs):
            g = e.gradient(self.vp, vs)
            return g["dk_vs"], g["residual"]

        def misfit(vs):
            return e.misfit(self.vp, vs)["residual"]

        vs1, _, info, self.f1 = iterate(self.vs, gradient, misfit, self.vsmin, self.vsmax, self.pur, self.f1)
        offset = self.offset
        if self.k > 1 and (info["residual"] - info["res0"]) / info["residual"] < self.err:  # SWD.m:330-333
            self.offset -= 3
            self.f1 = 0.5
        self.history.append(Step(k=self.k, offset=offset, offset_next=self.offset, **info))
        self.vs = vs1
        self.k += 1
        return self.history[-1]

    def run(self, iterations):
        """Up to `iterations` iterations; stops when the offset window reaches offmin (SWD.m:335)."""
        for _ in range(iterations):
            self.step()
            if self.offset == self.offmin:
                break
        return self.history

    def close(self):
        if self._eng is not None:
            self._eng.close()
            self._eng = None
