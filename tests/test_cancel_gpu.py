"""Cancelling calls in flight (swd_engine_cancel, swd_server_cancel of a running request).

Cancellation here needs no GPU fault: the engine's FD launches read a device word that the
cancel sets and return at once, and the call reports SWD_ERR_CANCELLED (5) on the host.  The
engine must be ready for the next call, with the same bits as before.
"""
import threading
import time

import numpy as np
import pytest

from swd_b200 import _lib, configs
from swd_b200.engine import GradientEngine
from swd_b200.serve import Server

pytestmark = pytest.mark.gpu

CANCELLED = 5


def _survey():
    return configs.batched_c2(ns=8, nt=4000)


def _run(e, s, out, key):
    try:
        out[key] = e.gradient(s.vp, s.vs)
    except _lib.SwdError as err:
        out[key] = err


def test_cancel_before_a_call_cancels_it_and_the_engine_recovers():
    s = configs.tiny(nt=400, ns=5)
    cr = np.ones((s.npair, s.ns))
    with GradientEngine(s) as e:
        e.set_observed(cr, cr)
        ref = e.gradient(s.vp, s.vs)
        e.cancel()
        with pytest.raises(_lib.SwdError) as err:
            e.gradient(s.vp, s.vs)
        assert err.value.status == CANCELLED and "cancelled" in str(err.value)
        again = e.gradient(s.vp, s.vs)  # graphs replayed with the word cleared
    for k in ("g_cl", "g_cm", "g_illum", "dk_vs", "cr_pre_r"):
        assert np.array_equal(again[k], ref[k]), k


def test_cancel_in_flight_stops_the_time_loops():
    s = _survey()
    cr = np.ones((s.npair, s.ns))
    with GradientEngine(s, snapshot_mode=1) as e:
        e.set_observed(cr, cr)
        ref = e.gradient(s.vp, s.vs)  # also captures the graphs
        t0 = time.perf_counter()
        e.gradient(s.vp, s.vs)
        full = time.perf_counter() - t0
        out = {}
        th = threading.Thread(target=_run, args=(e, s, out, "a"))
        t0 = time.perf_counter()
        th.start()
        time.sleep(full / 8)
        e.cancel()
        th.join()
        took = time.perf_counter() - t0
        if isinstance(out["a"], _lib.SwdError):
            assert out["a"].status == CANCELLED
            assert took < 0.8 * full, (took, full)
        else:  # the call ended before the cancel landed: the cancel applies to the next call
            with pytest.raises(_lib.SwdError):
                e.gradient(s.vp, s.vs)
        again = e.gradient(s.vp, s.vs)
    for k in ("g_cl", "g_cm", "g_illum", "cr_pre_r"):
        assert np.array_equal(again[k], ref[k]), k


def test_server_cancels_a_running_request():
    s = _survey()
    cr = np.ones((s.npair, s.ns))
    with Server(max_inflight=1) as srv:
        first = srv.submit(s, s.vp, s.vs, cr, cr, key=1)
        srv.wait(first)  # warm: engine and graphs built, kept idle under key 1
        rid = srv.submit(s, s.vp, s.vs, cr, cr, key=1)
        nxt = srv.submit(s, s.vp, s.vs, cr, cr, key=1)
        deadline = time.time() + 30
        while srv.stats()["admitted"] < 2 and time.time() < deadline:
            time.sleep(0.002)
        srv.cancel(rid)
        with pytest.raises(Exception, match="cancelled"):
            srv.wait(rid)
        o = srv.wait(nxt)  # the engine goes on with the next request
        st = srv.stats()
    assert st["cancelled"] >= 1 and np.isfinite(o["dk_vs"]).any()
