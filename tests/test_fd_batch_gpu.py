"""Several MEX-convention forward (swd_staggerfd_single_batch) or adjoint (swd_e2drtm_single_batch)
calls on grids of different sizes, advanced together by one launch per time step: every job's
outputs equal those of its own single call bit for bit, and those equal the oracle's."""
import dataclasses

import numpy as np
import pytest

import swd_b200 as S
from swd_b200 import configs
from swd_b200._lib import SwdError
from swd_b200.fd import eigen_e2drtm_single_batch, eigen_staggerfd_single_batch

pytestmark = pytest.mark.gpu


def _job(O, s, is_, src="w"):
    inp = O.fd_inputs(s.nbc, s.nt, s.dtx, s.dx, s.dt, int(s.sx[is_ - 1]), 1, s.gx, np.ones(s.ng), s.vp, s.vs,
                      source_type=src, in_wf=s.nt_wf)
    return inp, s.source()


def test_batch_of_grids_matches_separate_calls_and_oracle(O):
    tiny = configs.tiny(nt=400)
    c1 = dataclasses.replace(configs.plain_c1(), nt=800)
    cases = [(tiny, 2, "w"), (c1, 5, "w"), (tiny, 3, "p"), (c1, 11, "z")]  # different grids, nt, sources
    jobs, refs = [], []
    for s, is_, src in cases:
        inp, w = _job(O, s, is_, src)
        jobs.append((inp.iv, inp.temp, inp.ca, inp.cl, inp.cm, inp.cm1, inp.b, inp.b1, w))
        refs.append((inp, w))
    got = eigen_staggerfd_single_batch(jobs)
    for (inp, w), (su, sw, _), (s, is_, src) in zip(refs, got, cases):
        one = S.eigen_staggerfd_single(inp.iv, inp.temp, inp.ca, inp.cl, inp.cm, inp.cm1, inp.b, inp.b1, w,
                                       want_wf=False)
        assert np.abs(sw).max() > 0
        assert np.array_equal(sw, one[1]) and np.array_equal(su, one[0]), (s.name, is_, src)
        ref = O.mex_staggerfd(inp, w, want_wf=False)
        assert np.array_equal(sw, ref[1]) and np.array_equal(su, ref[0]), (s.name, is_, src)


def test_batch_wavefields_match_the_oracle(O):
    """With the strain wavefields: each job takes the snapshot variant on its own nt_wf steps
    (jobs with nt_wf 5 and 10 in one batch)."""
    tiny = configs.tiny(nt=400)
    c1 = dataclasses.replace(configs.plain_c1(), nt=800, nt_wf=10)
    jobs, refs = [], []
    for s, is_ in ((tiny, 1), (c1, 7)):
        inp, w = _job(O, s, is_)
        jobs.append((inp.iv, inp.temp, inp.ca, inp.cl, inp.cm, inp.cm1, inp.b, inp.b1, w))
        refs.append(O.mex_staggerfd(inp, w))
    for (su, sw, wf), ref in zip(eigen_staggerfd_single_batch(jobs, want_wf=True), refs):
        assert np.array_equal(sw, ref[1]) and np.array_equal(su, ref[0])
        for k in ("fux", "fuz", "bwx", "bwz"):
            assert np.abs(ref[2][k]).max() > 0
            assert np.array_equal(wf[k], ref[2][k]), k


def test_batch_rejects_a_bad_job_by_index(O):
    from swd_b200._lib import SwdError
    s = configs.tiny(nt=400)
    inp, w = _job(O, s, 1)
    bad = inp.iv.copy()
    bad[11] = 24  # fd_order 24 is not supported
    with pytest.raises(SwdError, match="job 1"):
        eigen_staggerfd_single_batch([(inp.iv, inp.temp, inp.ca, inp.cl, inp.cm, inp.cm1, inp.b, inp.b1, w),
                                      (bad, inp.temp, inp.ca, inp.cl, inp.cm, inp.cm1, inp.b, inp.b1, w)])


def test_adjoint_batch_matches_separate_calls_and_oracle(O):
    """Jobs with different grids, nt and nt_wf: each counts its steps back from its own nt and
    images on its own nt_wf steps; FP32 images as the single MEX accumulates them."""
    tiny = configs.tiny(nt=400)
    c1 = dataclasses.replace(configs.plain_c1(), nt=800, nt_wf=10)
    jobs, refs = [], []
    for s, is_ in ((tiny, 2), (c1, 4), (tiny, 3)):
        inp, w = _job(O, s, is_)
        _, sw, wf = O.mex_staggerfd(inp, w)
        res = np.asfortranarray(sw * 0.5)
        ai = O.fd_inputs(s.nbc, s.nt, s.dtx, s.dx, s.dt, int(s.sx[is_ - 1]), 1, s.gx, np.ones(s.ng), s.vp, s.vs,
                         in_wf=s.nt_wf, adjoint=True)
        args = (ai.iv, ai.temp, ai.ca, ai.cl, ai.cm, ai.cm1, ai.b, ai.b1, res, wf["fux"], wf["fuz"], wf["bwx"],
                wf["bwz"])
        jobs.append(args)
        refs.append((S.eigen_e2drtm_single(*args), O.mex_e2drtm(ai, res, wf, accum_fp64=False)))
    for got, (one, ref) in zip(eigen_e2drtm_single_batch(jobs), refs):
        for g, a, r in zip(got, one, ref):
            assert np.abs(r).max() > 0
            assert np.array_equal(g, a) and np.array_equal(g, r)


def test_gradient_of_several_surveys_in_one_batch(O):
    """swd_loop.gradient_many: the shots of two surveys on different grids go through one forward
    batch and one adjoint batch; each survey's gradient, picks and misfits equal its own
    swd_loop.gradient, bit for bit."""
    from swd_b200 import swd_loop
    cases = []
    for s in (configs.tiny(nt=400), dataclasses.replace(configs.plain_c1(), nt=1000)):
        cr0_r, cr0_l = O.observed_curves(s, s.vs_true)
        cases.append((s, s.vs, cr0_r, cr0_l))
    many = swd_loop.gradient_many(cases)
    for (s, vs, cr0_r, cr0_l), got in zip(cases, many):
        ref = swd_loop.gradient(s, vs, cr0_r, cr0_l)
        for k in ("g_cl", "g_cm", "g_illum", "cr_pre_r", "cr_pre_l"):
            assert np.array_equal(got[k], ref[k]), (s.name, k)
        for k in ("dk_vs", "res_r", "res_l"):
            assert np.array_equal(got[k], ref[k], equal_nan=True), (s.name, k)


def test_adjoint_batch_reads_the_kept_forward_snapshots(O):
    """swd_staggerfd_single_batch_keep / swd_e2drtm_single_batch_kept: the adjoint batch reads the
    forward batch's snapshots on the device and gives the images of the adjoint batch fed the
    forward's returned snapshots, bit for bit; the handle serves a second batch, and a job whose
    shape differs from its forward job's is refused before any launch."""
    tiny = configs.tiny(nt=400)
    c1 = dataclasses.replace(configs.plain_c1(), nt=800, nt_wf=10)
    fwd, adj_in = [], []
    for s, is_ in ((tiny, 2), (c1, 4)):
        inp, w = _job(O, s, is_)
        fwd.append((inp.iv, inp.temp, inp.ca, inp.cl, inp.cm, inp.cm1, inp.b, inp.b1, w))
        adj_in.append(O.fd_inputs(s.nbc, s.nt, s.dtx, s.dx, s.dt, int(s.sx[is_ - 1]), 1, s.gx, np.ones(s.ng), s.vp,
                                  s.vs, in_wf=s.nt_wf, adjoint=True))
    host = eigen_staggerfd_single_batch(fwd, want_wf=True)
    seis, kept = eigen_staggerfd_single_batch(fwd, keep=True)
    with_wf, on_device = [], []
    for (_, sw, wf), (_, sw2, wf2), ai in zip(host, seis, adj_in):
        assert np.array_equal(sw, sw2) and wf2 is None
        res = np.asfortranarray(sw * 0.5)
        head = (ai.iv, ai.temp, ai.ca, ai.cl, ai.cm, ai.cm1, ai.b, ai.b1, res)
        with_wf.append(head + (wf["fux"], wf["fuz"], wf["bwx"], wf["bwz"]))
        on_device.append(head + (None, None, None, None))
    want = eigen_e2drtm_single_batch(with_wf)
    for _ in range(2):
        for got, ref in zip(eigen_e2drtm_single_batch(on_device, kept), want):
            for g, r in zip(got, ref):
                assert np.abs(r).max() > 0 and np.array_equal(g, r)
    with pytest.raises(SwdError, match="job 0: the kept forward job"):
        eigen_e2drtm_single_batch(on_device[::-1], kept)
    with pytest.raises(ValueError, match="kept forward batch has 2 jobs"):
        eigen_e2drtm_single_batch(on_device[:1], kept)
