"""GPU parity of the FD kernels against the CPU oracle (bit-exact: same IEEE operations, no FMA)."""
import numpy as np
import pytest

from swd_b200 import configs
import swd_b200 as S

pytestmark = pytest.mark.gpu


def _inputs(O, survey, is_=1, single=True, adjoint=False, src="w"):
    s = survey
    return O.fd_inputs(s.nbc, s.nt, s.dtx, s.dx, s.dt, int(s.sx[is_ - 1]), 1, s.gx, np.ones(s.ng), s.vp, s.vs,
                       source_type=src, in_wf=s.nt_wf, single=single, adjoint=adjoint)


@pytest.mark.parametrize("single", [True, False])
def test_prep_model_matches_oracle(O, single):
    s = configs.plain_c1()
    m = S.prep_model(s.nbc, s.dtx, s.dx, s.dt, s.vp, s.vs, single=single)
    inp = _inputs(O, s, single=single)
    for k in ("temp", "ca", "cl", "cm", "cm1", "b", "b1"):
        assert np.array_equal(m[k], getattr(inp, k)), k


@pytest.mark.parametrize("src", ["w", "p", "s", "s1", "z"])
def test_staggerfd_single_bit_exact_tiny(O, src):
    s = configs.tiny(nt=400)
    inp = _inputs(O, s, 2, src=src)
    w = s.source()
    ref = O.mex_staggerfd(inp, w)
    got = S.eigen_staggerfd_single(inp.iv, inp.temp, inp.ca, inp.cl, inp.cm, inp.cm1, inp.b, inp.b1, w)
    assert np.array_equal(got[1], ref[1]) and np.array_equal(got[0], ref[0])
    for k in ("fux", "fuz", "bwx", "bwz"):
        assert np.array_equal(got[2][k], ref[2][k]), k


def test_staggerfd_single_bit_exact_plain_30x120(O):
    s = configs.plain_c1()
    inp = _inputs(O, s, 5)
    w = s.source()
    ref = O.mex_staggerfd(inp, w)
    got = S.eigen_staggerfd_single(inp.iv, inp.temp, inp.ca, inp.cl, inp.cm, inp.cm1, inp.b, inp.b1, w)
    assert np.abs(ref[1]).max() > 0
    assert np.array_equal(got[1], ref[1])
    for k in ("fux", "fuz", "bwx", "bwz"):
        assert np.array_equal(got[2][k], ref[2][k]), k


def test_staggerfd_double_bit_exact(O):
    s = configs.tiny(nt=400)
    inp = _inputs(O, s, 3, single=False)
    w = s.source()
    ref = O.mex_staggerfd(inp, w)
    got = S.eigen_staggerfd_double(inp.iv, inp.temp, inp.ca, inp.cl, inp.cm, inp.cm1, inp.b, inp.b1, w)
    assert np.array_equal(got[1], ref[1])
    for k in ("fux", "fuz", "bwx", "bwz"):
        assert np.array_equal(got[2][k], ref[2][k]), k


@pytest.mark.parametrize("survey", ["tiny", "plain"])
def test_e2drtm_single_bit_exact(O, survey):
    s = configs.tiny(nt=400) if survey == "tiny" else configs.plain_c1()
    inp = _inputs(O, s, 2)
    ainp = _inputs(O, s, 2, adjoint=True)
    _, sw, wf = O.mex_staggerfd(inp, s.source())
    res = np.asfortranarray(np.random.default_rng(0).standard_normal(sw.shape).astype(np.float32) * 1e-3)
    ref = O.mex_e2drtm(ainp, res, wf, accum_fp64=True)
    got = S.eigen_e2drtm_single(ainp.iv, ainp.temp, ainp.ca, ainp.cl, ainp.cm, ainp.cm1, ainp.b, ainp.b1, res,
                                wf["fux"], wf["fuz"], wf["bwx"], wf["bwz"], fp64_out=True)
    for g, r in zip(got, ref):
        assert np.abs(r).max() > 0
        assert np.array_equal(g, r)
    # single images accumulate in FP32, as the reference's single MEX does
    ref32 = O.mex_e2drtm(ainp, res, wf, accum_fp64=False)
    got32 = S.eigen_e2drtm_single(ainp.iv, ainp.temp, ainp.ca, ainp.cl, ainp.cm, ainp.cm1, ainp.b, ainp.b1, res,
                                  wf["fux"], wf["fuz"], wf["bwx"], wf["bwz"])
    for g, r in zip(got32, ref32):
        assert g.dtype == np.float32 and np.array_equal(g, r.astype(np.float32))


def test_e2drtm_double_bit_exact(O):
    s = configs.tiny(nt=400)
    inp = _inputs(O, s, 1, single=False)
    ainp = _inputs(O, s, 1, single=False, adjoint=True)
    _, sw, wf = O.mex_staggerfd(inp, s.source())
    res = np.asfortranarray(np.random.default_rng(1).standard_normal(sw.shape))
    ref = O.mex_e2drtm(ainp, res, wf)
    got = S.eigen_e2drtm_double(ainp.iv, ainp.temp, ainp.ca, ainp.cl, ainp.cm, ainp.cm1, ainp.b, ainp.b1, res,
                                wf["fux"], wf["fuz"], wf["bwx"], wf["bwz"])
    for g, r in zip(got, ref):
        assert np.array_equal(g, r)


def test_m_level_wrappers_match_oracle(O):
    s = configs.tiny(nt=400)
    w = s.source().astype(np.float32)
    su, sw, www = S.staggerfd_eigen(1, s.nbc, s.nt, s.dtx, s.dx, s.dt, 5, 1, s.gx, np.ones(s.ng), w, s.vp, s.vs)
    rsu, rsw, rw = O.staggerfd_eigen(1, s.nbc, s.nt, s.dtx, s.dx, s.dt, 5, 1, s.gx, np.ones(s.ng), w, s.vp, s.vs)
    assert np.array_equal(sw, rsw)
    res = np.asfortranarray(sw * 0.5)
    got = S.e2drtm_eigen(www, res, 1, s.nbc, s.nt, s.dtx, s.dx, s.dt, s.gx, np.ones(s.ng), w, s.vp, s.vs,
                         fp64_out=True)
    ref = O.e2drtm_eigen(rw, res, 1, s.nbc, s.nt, s.dtx, s.dx, s.dt, s.gx, np.ones(s.ng), w, s.vp, s.vs)
    for g, r in zip(got, ref):
        assert np.array_equal(g, r)
