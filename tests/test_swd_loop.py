"""The per-shot SWD.m loop on the MEX-convention entry points (swd_b200.swd_loop)."""
import numpy as np
import pytest

from swd_b200 import configs, swd_loop


def test_smooth2a_and_side_rules_match_the_oracle(O):
    a = np.random.default_rng(4).standard_normal((9, 17))
    a[3, 5] = np.nan
    np.testing.assert_allclose(swd_loop.smooth2a(a, 1, 2), O.smooth2a(a, 1, 2), rtol=1e-12, atol=1e-15,
                               equal_nan=True)
    for ns, m, M, w in [(12, 0, 10, 3), (96, 0, 6, 3), (5, 2, 4, 3), (40, 0, 2, 3)]:
        for is_ in range(1, ns + 1):
            assert swd_loop.has_right(is_, ns, m, M, w) == O.has_right(is_, ns, m, M, w)
            assert swd_loop.has_left(is_, m, M, w) == O.has_left(is_, m, M, w)


@pytest.mark.gpu
def test_fp64_loop_matches_the_fp64_oracle(O):
    """SWD.m's double path: FP64 FD bit-exact, spectra to 1e-9, so picks identical and the
    gradient within 1e-9 (relative L2)."""
    s = configs.tiny(nt=400, ns=5)
    cr0_r, cr0_l = O.observed_curves(s, s.vs_true)
    ref = O.gradient(s, s.vs, cr0_r, cr0_l, single=False)
    got = swd_loop.gradient(s, s.vs, cr0_r, cr0_l, single=False)
    assert np.array_equal(got["cr_pre_r"], ref["cr_pre_r"]) and np.array_equal(got["cr_pre_l"], ref["cr_pre_l"])
    for k in ("g_cl", "g_cm", "g_illum", "dk_vs"):
        assert np.linalg.norm(got[k] - ref[k]) / np.linalg.norm(ref[k]) < 1e-9, k
    assert got["residual"] == pytest.approx(ref["residual"], rel=1e-12)


@pytest.mark.gpu
def test_fp32_loop_matches_the_batched_engine():
    """The per-shot FP32 loop and the batched engine: identical picks and misfits, images
    within the FP32-rounding tolerance of the adjoint source (1e-6)."""
    from swd_b200.engine import GradientEngine
    s = configs.tiny(nt=400, ns=5)
    with GradientEngine(s) as e:
        cr0_r, cr0_l = e.observed_curves(s.vp_true, s.vs_true)
        e.set_observed(cr0_r, cr0_l)
        eng = e.gradient(s.vp, s.vs)
    got = swd_loop.gradient(s, s.vs, cr0_r, cr0_l, single=True)
    assert np.array_equal(got["cr_pre_r"], eng["cr_pre_r"]) and np.array_equal(got["cr_pre_l"], eng["cr_pre_l"])
    np.testing.assert_allclose(got["res_r"], eng["res_r"], rtol=1e-12, equal_nan=True)
    for k in ("g_cl", "g_cm", "g_illum", "dk_vs"):
        assert np.linalg.norm(got[k] - eng[k]) / np.linalg.norm(eng[k]) < 1e-6, k
