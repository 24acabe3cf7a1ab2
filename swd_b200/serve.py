"""Served request loop on one GPU (swd_server_* of libswd.so).

    srv = Server(max_inflight=4)
    rid = srv.submit(survey, vp, vs, cr0_r, cr0_l, kind="gradient", key=7)
    out = srv.wait(rid)          # dict: dk_vs, res_r, res_l, cr_pre_r, cr_pre_l, residual, timings

Requests of any grid size and shot count are admitted in arrival order when a slot is free and
their engine's planned HBM fits; requests in flight overlap on the device.  Requests that share
a nonzero key (the iterations of one inversion) reuse the resident engine of that survey.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import call
from .engine import EngineInfo, EngineOpts, SurveyC, _bind as _bind_engine, survey_struct

_dp = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p

KIND = {"gradient": 0, "misfit": 1}


class ServerOpts(ctypes.Structure):
    _fields_ = [("hbm_budget", ctypes.c_size_t), ("max_inflight", ctypes.c_int), ("device", ctypes.c_int),
                ("keep_engines", ctypes.c_int)]


class Request(ctypes.Structure):
    _fields_ = [("survey", ctypes.POINTER(SurveyC)), ("survey_key", ctypes.c_uint64), ("kind", ctypes.c_int),
                ("npair", ctypes.c_int), ("wavelet", _dp), ("vp", _dp), ("vs", _dp), ("cr0_r", _dp),
                ("cr0_l", _dp)]


class Result(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("residual", ctypes.c_double), ("queue_ms", ctypes.c_double),
                ("run_ms", ctypes.c_double), ("total_ms", ctypes.c_double), ("reused_engine", ctypes.c_int),
                ("engine_bytes", ctypes.c_size_t), ("dk_vs", _dp), ("res_r", _dp), ("res_l", _dp),
                ("cr_pre_r", _dp), ("cr_pre_l", _dp)]


class Stats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("admitted", ctypes.c_uint64), ("completed", ctypes.c_uint64),
                ("cancelled", ctypes.c_uint64), ("waits_for_memory", ctypes.c_uint64),
                ("peak_inflight", ctypes.c_int), ("idle_engines", ctypes.c_int), ("peak_bytes", ctypes.c_size_t),
                ("bytes_in_use", ctypes.c_size_t), ("budget", ctypes.c_size_t)]


SERVER_SYMBOLS = ["swd_engine_plan", "swd_server_create", "swd_server_submit", "swd_server_wait",
                  "swd_server_cancel", "swd_server_stats", "swd_server_destroy"]


def _bind():
    L = _bind_engine()
    if getattr(L, "_server_bound", False):
        return L
    sigs = {
        "swd_engine_plan": [ctypes.POINTER(SurveyC), ctypes.POINTER(EngineOpts), ctypes.POINTER(EngineInfo)],
        "swd_server_create": [ctypes.POINTER(ServerOpts), ctypes.POINTER(_vp)],
        "swd_server_submit": [_vp, ctypes.POINTER(Request), ctypes.POINTER(ctypes.c_uint64)],
        "swd_server_wait": [_vp, ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(Result)],
        "swd_server_cancel": [_vp, ctypes.c_uint64],
        "swd_server_stats": [_vp, ctypes.POINTER(Stats)],
        "swd_server_destroy": [_vp],
    }
    for n, a in sigs.items():
        f = getattr(L, n)
        f.argtypes = a
        f.restype = ctypes.c_int
    L._server_bound = True
    return L


def plan(survey, hbm_budget=0, **opts):
    """The engine plan (batch, mode, bytes, npair ...) for a survey, without allocating."""
    _bind()
    sc = survey_struct(survey)
    o = EngineOpts(int(hbm_budget), *[int(opts.get(k, 0)) for k, _ in EngineOpts._fields_[1:]])
    inf = EngineInfo()
    call("swd_engine_plan", ctypes.byref(sc), ctypes.byref(o), ctypes.byref(inf))
    return {k: getattr(inf, k) for k, _ in EngineInfo._fields_}


def _f(a):
    return np.asfortranarray(np.asarray(a, np.float64))


class Server:
    def __init__(self, hbm_budget=0, max_inflight=4, device=0, keep_engines=True):
        _bind()
        h = _vp()
        call("swd_server_create", ctypes.byref(ServerOpts(int(hbm_budget), int(max_inflight), int(device),
                                                          int(keep_engines))), ctypes.byref(h))
        self._h = h
        self._pending = {}

    def submit(self, survey, vp, vs, cr0_r, cr0_l, kind="gradient", key=0, wavelet=None):
        sc = survey_struct(survey)
        npair = int(np.asarray(cr0_r).shape[0])
        arrs = [np.ascontiguousarray(np.asarray(survey.source() if wavelet is None else wavelet, np.float64)),
                _f(vp), _f(vs), _f(cr0_r), _f(cr0_l)]
        if arrs[3].shape != (npair, survey.ns) or arrs[4].shape != (npair, survey.ns):
            raise ValueError("cr0_r / cr0_l must be npair x ns")
        q = Request(ctypes.pointer(sc), int(key), KIND[kind], npair, *[a.ctypes.data_as(_dp) for a in arrs])
        rid = ctypes.c_uint64()
        call("swd_server_submit", self._h, ctypes.byref(q), ctypes.byref(rid))
        self._pending[rid.value] = (survey, npair, kind)
        return rid.value

    def wait(self, rid, timeout_ms=-1):
        survey, npair, kind = self._pending[rid]
        ns, shp = survey.ns, (survey.nz, survey.nx)
        out = {"res_r": np.zeros(ns), "res_l": np.zeros(ns), "cr_pre_r": np.zeros((npair, ns), order="F"),
               "cr_pre_l": np.zeros((npair, ns), order="F")}
        if kind == "gradient":
            out["dk_vs"] = np.zeros(shp, order="F")
        r = Result()
        for k in ("dk_vs", "res_r", "res_l", "cr_pre_r", "cr_pre_l"):
            if k in out:
                setattr(r, k, out[k].ctypes.data_as(_dp))
        rc = _lib.lib().swd_server_wait(self._h, rid, int(timeout_ms), ctypes.byref(r))
        if rc == 7:  # SWD_ERR_TIMEOUT: still pending
            return None
        del self._pending[rid]
        if rc != 0:
            raise _lib.SwdError("swd_server_wait", rc, _lib.lib().swd_last_error().decode())
        out.update(residual=r.residual, queue_ms=r.queue_ms, run_ms=r.run_ms, total_ms=r.total_ms,
                   reused_engine=bool(r.reused_engine), engine_bytes=r.engine_bytes)
        return out

    def cancel(self, rid):
        call("swd_server_cancel", self._h, rid)

    def stats(self):
        s = Stats()
        call("swd_server_stats", self._h, ctypes.byref(s))
        return {k: getattr(s, k) for k, _ in Stats._fields_}

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().swd_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
