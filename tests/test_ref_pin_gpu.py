"""The CUDA FD path against the reference's own MEX sources (oracle/_ref), bit for bit.

oracle/_ref is core/eigen_staggerfd_single.cpp and core/eigen_e2drtm_single.cpp compiled
unmodified against the Eigen / MEX API stand-ins in oracle/ref_shim.  These tests call the
C-ABI's MEX-convention entry points (swd_staggerfd_single / swd_e2drtm_single, the calls a
MEX shim makes) and the batched engine's default kernels, and compare with it directly.
"""
import numpy as np
import pytest

import swd_b200 as S
from swd_b200 import configs

pytestmark = pytest.mark.gpu


def _inp(O, s, sx, adjoint=False):
    return O.fd_inputs(s.nbc, s.nt, s.dtx, s.dx, s.dt, sx, 1, s.gx, np.ones(s.ng), s.vp, s.vs,
                       in_wf=s.nt_wf, adjoint=adjoint)


def _mex_pair(O, R, s, sx, w, res_scale, seed):
    inp = _inp(O, s, sx)
    got = S.eigen_staggerfd_single(inp.iv, inp.temp, inp.ca, inp.cl, inp.cm, inp.cm1, inp.b, inp.b1, w)
    ref = R.mex_staggerfd(inp, w)
    assert np.abs(ref[1]).max() > 0
    assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1])
    for k in ("fux", "fuz", "bwx", "bwz"):
        assert np.array_equal(got[2][k], ref[2][k]), k
    ainp = _inp(O, s, 0, adjoint=True)
    res = np.asfortranarray(np.random.default_rng(seed).standard_normal(ref[1].shape).astype(np.float32)
                            * np.float32(res_scale))
    gi = S.eigen_e2drtm_single(ainp.iv, ainp.temp, ainp.ca, ainp.cl, ainp.cm, ainp.cm1, ainp.b, ainp.b1, res,
                               ref[2]["fux"], ref[2]["fuz"], ref[2]["bwx"], ref[2]["bwz"])
    ri = R.mex_e2drtm(ainp, res, ref[2])
    for g, r in zip(gi, ri):
        assert np.abs(r).max() > 0
        assert g.dtype == np.float32 and np.array_equal(g, r)


def test_mex_calls_match_the_reference_30x120(O, R):
    s = configs.plain_c1()
    _mex_pair(O, R, s, int(s.sx[3]), s.source(), 1e-3, 1)


def test_mex_calls_match_the_reference_100x600_grid(O, R):
    s = configs.batched_c2(ns=4, nt=1000)
    w = np.random.default_rng(11).standard_normal(s.nt).astype(np.float32)
    _mex_pair(O, R, s, 1 + 6 * 40, w, 1e-2, 2)


def test_mex_calls_match_the_reference_400x3000_grid(O, R):
    s = configs.large_c5(ns=2, nt=100)
    w = np.random.default_rng(12).standard_normal(s.nt).astype(np.float32)
    _mex_pair(O, R, s, int(s.sx[1]), w, 1e-2, 3)


@pytest.mark.parametrize("survey", ["tiny", "plain"])
def test_engine_gradient_matches_the_reference_shot_loop(O, R, survey):
    """The batched engine (default two-steps-per-launch kernels, FP32 per-shot image sums as the
    single MEX) against SWD_single.m's shot loop run on the reference's own FD.  Picks are
    identical.  The adjoint source goes through the GPU's FP64 direct DFT and the oracle's FFT,
    which differ by ~1e-13 and can flip the FP32 rounding of a few adjoint-source samples
    (SWD_single.m:193), so the image sums are compared at 1e-6 relative L2, and exactly where
    no sample flips (the tiny survey)."""
    from swd_b200.engine import GradientEngine
    s = configs.tiny(nt=400, ns=5) if survey == "tiny" else configs.plain_c1(ns=4, nt=1500)
    cr0_r, cr0_l = O.observed_curves(s, s.vs_true)
    ref = O.gradient(s, s.vs, cr0_r, cr0_l, fd="reference")
    with GradientEngine(s) as e:
        e.set_observed(cr0_r, cr0_l)
        out = e.gradient(s.vp, s.vs)
    assert np.array_equal(out["cr_pre_r"], ref["cr_pre_r"]) and np.array_equal(out["cr_pre_l"], ref["cr_pre_l"])
    for k in ("g_cl", "g_cm", "g_illum", "dk_vs"):
        if survey == "tiny":
            assert np.array_equal(out[k], ref[k]), k
        else:
            assert np.linalg.norm(out[k] - ref[k]) / np.linalg.norm(ref[k]) < 1e-6, k
