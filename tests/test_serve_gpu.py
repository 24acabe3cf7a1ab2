"""The served request loop: concurrent requests of different surveys give the same results as
each request run alone on its own engine; admission by memory, engine reuse and cancellation."""
import numpy as np
import pytest

from swd_b200 import configs
from swd_b200.engine import GradientEngine
from swd_b200.serve import Server, plan

pytestmark = pytest.mark.gpu


def _surveys():
    a = configs.tiny(nt=400, ns=5)
    b = configs.tiny(nz=10, nx=32, nbc=6, nt=400, ns=4, seed=5)
    c = configs.plain_c1(ns=4, nt=2000)
    return [a, b, c]


def _cr0(s, seed):
    r = np.random.default_rng(seed)
    return (s.vmin + r.integers(5, 60, (s.npair, s.ns))).astype(float), np.ones((s.npair, s.ns))


def _alone(s, cr0_r, cr0_l, kind, vs):
    with GradientEngine(s) as e:
        e.set_observed(cr0_r, cr0_l)
        return e.gradient(s.vp_ratio * vs, vs) if kind == "gradient" else e.misfit(s.vp_ratio * vs, vs)


def test_requests_in_the_mix_match_requests_alone():
    ss = _surveys()
    jobs = []
    for i in range(8):
        s = ss[i % 3]
        vs = s.vs * (1.0 + 0.01 * i)
        cr0_r, cr0_l = _cr0(s, i)
        kind = "gradient" if i % 4 != 3 else "misfit"
        jobs.append((s, vs, cr0_r, cr0_l, kind, 1 + i % 3))
    with Server(max_inflight=3) as srv:
        ids = [srv.submit(s, s.vp_ratio * vs, vs, r, l, kind=k, key=key) for s, vs, r, l, k, key in jobs]
        outs = [srv.wait(i) for i in ids]
        st = srv.stats()
    assert st["completed"] == 8 and st["peak_inflight"] >= 2
    assert any(o["reused_engine"] for o in outs)
    for (s, vs, r, l, k, _), o in zip(jobs, outs):
        ref = _alone(s, r, l, k, vs)
        np.testing.assert_array_equal(o["cr_pre_r"], ref["cr_pre_r"])
        np.testing.assert_array_equal(o["cr_pre_l"], ref["cr_pre_l"])
        np.testing.assert_array_equal(o["res_r"], ref["res_r"])
        assert o["residual"] == ref["residual"] or (np.isnan(o["residual"]) and np.isnan(ref["residual"]))
        if k == "gradient":
            np.testing.assert_array_equal(o["dk_vs"], ref["dk_vs"])


def test_admission_waits_for_memory_and_cancels():
    s = configs.plain_c1(ns=4, nt=2000)
    need = plan(s, hbm_budget=8 << 30)["bytes"]
    cr0_r, cr0_l = _cr0(s, 1)
    with Server(hbm_budget=int(need * 1.6), max_inflight=1, keep_engines=False) as srv:
        ids = [srv.submit(s, s.vp, s.vs, cr0_r, cr0_l, kind="misfit") for _ in range(3)]
        srv.cancel(ids[2])
        a, b = srv.wait(ids[0]), srv.wait(ids[1])
        with pytest.raises(Exception, match="cancelled"):
            srv.wait(ids[2])
        np.testing.assert_array_equal(a["cr_pre_r"], b["cr_pre_r"])
        assert b["queue_ms"] > 0
    with Server(hbm_budget=need // 4, max_inflight=1) as srv:
        rid = srv.submit(s, s.vp, s.vs, cr0_r, cr0_l)
        with pytest.raises(Exception):
            srv.wait(rid)
