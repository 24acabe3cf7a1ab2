"""The oracle's FD loops against the reference's own MEX sources (CPU).

``oracle/_ref`` is core/eigen_staggerfd_single.cpp and core/eigen_e2drtm_single.cpp
compiled unmodified (Eigen / MEX API stand-ins in oracle/ref_shim).  The restated oracle
(oracle/swd_oracle.cpp) must give the same bits: seismograms, the four snapshot fields and
the three FP32 images, on the tiny, 30 x 120, 100 x 600 and 400 x 3000 grids.  The GPU
tests compare the CUDA path with the oracle, so this pins them to the reference too
(tests/test_ref_pin_gpu.py also compares the GPU with oracle/_ref directly).
"""
import numpy as np
import pytest

from swd_b200 import configs


def _inp(O, s, sx, adjoint=False, src="w"):
    return O.fd_inputs(s.nbc, s.nt, s.dtx, s.dx, s.dt, sx, 1, s.gx, np.ones(s.ng), s.vp, s.vs,
                       source_type=src, in_wf=s.nt_wf, adjoint=adjoint)


def _noise(shape, seed, scale):
    return np.asfortranarray(np.random.default_rng(seed).standard_normal(shape).astype(np.float32) * np.float32(scale))


def _check_forward(O, R, inp, w):
    su, sw, wf = O.mex_staggerfd(inp, w)
    ru, rw, rwf = R.mex_staggerfd(inp, w)
    assert np.abs(rw).max() > 0
    assert np.array_equal(su, ru) and np.array_equal(sw, rw)
    for k in ("fux", "fuz", "bwx", "bwz"):
        assert np.abs(rwf[k]).max() > 0, k
        assert np.array_equal(wf[k], rwf[k]), k
    return sw, wf


def _check_adjoint(O, R, ainp, res, wf):
    got = O.mex_e2drtm(ainp, res, wf, accum_fp64=False)
    ref = R.mex_e2drtm(ainp, res, wf)
    for g, r in zip(got, ref):
        assert np.abs(r).max() > 0
        assert np.array_equal(g, r.astype(np.float64))


@pytest.mark.parametrize("src", ["w", "p", "s", "s1", "z"])
def test_every_source_type_tiny(O, R, src):
    """source_type 1..5 of core/eigen_staggerfd_single.cpp:285-300 (5, 'w', is what SWD uses)."""
    s = configs.tiny(nt=400)
    inp = _inp(O, s, int(s.sx[1]), src=src)
    sw, wf = _check_forward(O, R, inp, s.source())
    _check_adjoint(O, R, _inp(O, s, 0, adjoint=True), _noise(sw.shape, 5, 1e-3), wf)


def test_plain_30x120_full_length(O, R):
    """The 30 x 120 survey (52 x 160 padded, nt 6000): one shot through both MEX calls, the
    adjoint driven by the forward seismogram as in SWD's own flow."""
    s = configs.plain_c1()
    inp = _inp(O, s, int(s.sx[4]))
    sw, wf = _check_forward(O, R, inp, s.source())
    _check_adjoint(O, R, _inp(O, s, 0, adjoint=True), np.asfortranarray(sw * np.float32(0.25)), wf)


@pytest.mark.parametrize("sx", [1, 301, 600])
def test_100x600_grid(O, R, sx):
    """The 100 x 600 survey's grid (132 x 660 padded, 600 receivers) for 800 steps with a seeded
    random source signal (the Ricker pulse barely starts in 800 steps), sources at both edges and
    in the middle, and a random adjoint source."""
    s = configs.batched_c2(ns=4, nt=800)
    w = np.random.default_rng(sx).standard_normal(s.nt).astype(np.float32)
    inp = _inp(O, s, sx)
    sw, wf = _check_forward(O, R, inp, w)
    _check_adjoint(O, R, _inp(O, s, 0, adjoint=True), _noise(sw.shape, sx, 1e-2), wf)


def test_400x3000_grid(O, R):
    """The 400 x 3000 survey's grid (442 x 3080 padded, 1200 receivers every second column) for
    60 steps with a random source signal and adjoint source."""
    s = configs.large_c5(ns=2, nt=60)
    w = np.random.default_rng(7).standard_normal(s.nt).astype(np.float32)
    inp = _inp(O, s, int(s.sx[1]))
    sw, wf = _check_forward(O, R, inp, w)
    _check_adjoint(O, R, _inp(O, s, 0, adjoint=True), _noise(sw.shape, 8, 1e-2), wf)


def test_shot_loop_on_the_reference_fd(O, R):
    """The oracle's SWD_single.m shot loop run on the reference's own FD (fd='reference') gives
    the same picks, misfits and FP32 image sums as on the restated FD."""
    s = configs.tiny(nt=400, ns=5)
    cr0_r, cr0_l = O.observed_curves(s, s.vs_true)
    a = O.gradient(s, s.vs, cr0_r, cr0_l)
    b = O.gradient(s, s.vs, cr0_r, cr0_l, fd="reference")
    for k in ("cr_pre_r", "cr_pre_l", "g_cl", "g_cm", "g_illum", "dk_vs"):
        assert np.array_equal(a[k], b[k]), k
    np.testing.assert_array_equal(a["res_r"], b["res_r"])


def test_a_changed_operation_is_caught(O, R):
    """The comparison is sharp: the restated forward loop with one input field nudged by one
    FP32 ulp on a single cell no longer matches the reference bit for bit."""
    s = configs.tiny(nt=400)
    inp = _inp(O, s, int(s.sx[1]))
    w = s.source()
    _, rw, _ = R.mex_staggerfd(inp, w)
    z, x = inp.nzbc // 2, inp.nxbc // 2
    inp.ca[z, x] = np.nextafter(inp.ca[z, x], np.float32(np.inf))
    _, sw, _ = O.mex_staggerfd(inp, w)
    assert not np.array_equal(sw, rw)
