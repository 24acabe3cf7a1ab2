"""Batched gradient engine: the per-iteration shot loops of SWD.m on the GPU.

    GradientEngine.observed_curves  SWD.m:150-162  (RTr/RTl + LHDispPick of the observed data)
    GradientEngine.gradient         SWD.m:171-201  (forward, spectra, picks, ADWDgrad_1, adjoint,
                                                     shot sum, illumination, smoothing)
    GradientEngine.misfit           SWD.m:215-228  (forward-only misfit of a trial model)

All shots of an iteration run batched through libswd.so; models are MATLAB
nz x nx arrays (column-major numpy, or device tensors for gradient_device).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import call, ptr

_i = ctypes.c_int
_d = ctypes.c_double
_ip = ctypes.POINTER(ctypes.c_int)
_dp = ctypes.POINTER(ctypes.c_double)


class SurveyC(ctypes.Structure):
    """swd_survey of include/swd.h."""
    _fields_ = [("nz", _i), ("nx", _i), ("nbc", _i), ("nt", _i), ("nt_wf", _i), ("fd_order", _i), ("isfs", _i),
                ("source_type", _i), ("dx", _d), ("dt", _d), ("ns", _i), ("sx", _ip), ("sz", _ip), ("ng", _i),
                ("gx0", _i), ("dgx", _i), ("gz", _i), ("df", _d), ("fmin", _d), ("fmax", _d), ("vmin", _d),
                ("vmax", _d), ("dv", _d), ("offset", _i), ("m", _i), ("M", _i), ("w", _i), ("ini", _i),
                ("pick_method", _i), ("soft_arg_norm", _d), ("smooth_z", _i), ("smooth_x", _i),
                ("shot_no", _ip), ("ns_total", _i)]


class EngineOpts(ctypes.Structure):
    _fields_ = [("hbm_budget", ctypes.c_size_t), ("max_batch", _i), ("snapshot_mode", _i), ("ckpt_interval", _i),
                ("use_graphs", _i), ("chunk_rows", _i), ("device", _i), ("warps", _i), ("cells", _i),
                ("ring_fwd", _i), ("ring_adj", _i), ("autotune", _i), ("radon_precision", _i),
                ("fd_schedule", _i), ("adjoint_weight", _i), ("image_precision", _i)]


class EngineInfo(ctypes.Structure):
    _fields_ = [("batch", _i), ("nbatch", _i), ("mode", _i), ("ckpt_interval", _i), ("bytes", ctypes.c_size_t),
                ("npair", _i), ("np", _i), ("ccn", _i), ("nzbc", _i), ("nxbc", _i), ("chunk_rows", _i),
                ("warps", _i), ("cells", _i), ("ring_fwd", _i), ("ring_adj", _i), ("tuned_fwd_us", _d),
                ("tuned_adj_us", _d), ("fd_schedule", _i)]


class GradientOut(ctypes.Structure):
    _fields_ = [("g_cl", _dp), ("g_cm", _dp), ("g_illum", _dp), ("dk_vs", _dp), ("res_r", _dp), ("res_l", _dp),
                ("cr_pre_r", _dp), ("cr_pre_l", _dp), ("residual", _d)]


_SRC = {"p": 1, "s": 2, "s1": 3, "z": 4, "w": 5}
_RPREC = {"fp64": 0, "bf16x2": 2, "bf16x3": 3}


def _bind():
    L = _lib.lib()
    if getattr(L, "_engine_bound", False):
        return L
    vp = ctypes.c_void_p
    sigs = {
        "swd_engine_create": [ctypes.POINTER(SurveyC), ctypes.POINTER(EngineOpts), ctypes.POINTER(vp)],
        "swd_engine_destroy": [vp],
        "swd_engine_info": [vp, ctypes.POINTER(EngineInfo)],
        "swd_engine_set_source": [vp, _dp],
        "swd_engine_set_observed": [vp, _dp, _dp],
        "swd_engine_observed_curves": [vp, _dp, _dp, _dp, _dp],
        "swd_engine_misfit": [vp, _dp, _dp, _dp, _dp, _dp, _dp, _dp],
        "swd_engine_gradient": [vp, _dp, _dp, ctypes.POINTER(GradientOut)],
        "swd_engine_gradient_device": [vp, vp, vp, vp, _dp],
        "swd_engine_stream": [vp, ctypes.POINTER(vp)],
        "swd_engine_cancel": [vp],
        "swd_engine_cancel_clear": [vp],
        "swd_engine_radon_stats": [vp, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)],
        "swd_engine_shot_sums_device": [vp, vp, vp, vp, _dp, _ip],
        "swd_engine_assemble_device": [vp, vp, vp],
        "swd_engine_set_timing": [vp, _i],
        "swd_engine_phase_times": [vp, _dp, _dp, _dp],
    }
    for n, a in sigs.items():
        f = getattr(L, n)
        f.argtypes = a
        f.restype = ctypes.c_int
    L._engine_bound = True
    return L


ENGINE_SYMBOLS = ["swd_engine_create", "swd_engine_destroy", "swd_engine_info", "swd_engine_set_source",
                  "swd_engine_set_observed", "swd_engine_observed_curves", "swd_engine_misfit",
                  "swd_engine_gradient", "swd_engine_gradient_device", "swd_engine_stream",
                  "swd_engine_shot_sums_device", "swd_engine_assemble_device", "swd_engine_set_timing",
                  "swd_engine_phase_times", "swd_engine_cancel", "swd_engine_cancel_clear",
                  "swd_engine_radon_stats"]


def survey_struct(s):
    """swd_survey for a configs.Survey (keeps the position arrays alive on the struct)."""
    sx = np.ascontiguousarray(np.asarray(s.sx, np.int32))
    sz = np.ascontiguousarray(np.ones(s.ns, np.int32))
    gx = np.asarray(s.gx)
    shot_no = None if s.shot_no is None else np.ascontiguousarray(np.asarray(s.shot_no, np.int32))
    c = SurveyC(nz=s.nz, nx=s.nx, nbc=s.nbc, nt=s.nt, nt_wf=s.nt_wf, fd_order=s.fd_order, isfs=s.isfs,
                source_type=_SRC[s.source_type], dx=s.dx, dt=s.dt, ns=s.ns, sx=sx.ctypes.data_as(_ip),
                sz=sz.ctypes.data_as(_ip), ng=s.ng, gx0=int(gx[0]), dgx=int(gx[1] - gx[0]), gz=1, df=s.df,
                fmin=s.fmin, fmax=s.fmax, vmin=s.vmin, vmax=s.vmax, dv=s.dv, offset=s.offset, m=s.m, M=s.M, w=s.w,
                ini=s.ini, pick_method=1, soft_arg_norm=s.soft_arg_norm, smooth_z=s.smooth_z, smooth_x=s.smooth_x,
                shot_no=shot_no.ctypes.data_as(_ip) if shot_no is not None else None, ns_total=int(s.ns_total))
    c._keep = (sx, sz, shot_no)
    return c


def _f(a):
    return np.asfortranarray(np.asarray(a, np.float64))


class GradientEngine:
    """Owns device memory, CUDA graphs and the plan for one survey."""

    def __init__(self, survey, hbm_budget=0, max_batch=0, snapshot_mode=0, ckpt_interval=0, use_graphs=True,
                 chunk_rows=0, device=0, source=None, warps=0, cells=0, ring_fwd=0, ring_adj=0, autotune=False,
                 radon_precision="fp64", fd_schedule=0, adjoint_weight="softmax", image_precision="fp32"):
        L = _bind()
        self.survey = survey
        self._sc = survey_struct(survey)
        opts = EngineOpts(int(hbm_budget), int(max_batch), int(snapshot_mode), int(ckpt_interval), int(use_graphs),
                          int(chunk_rows), int(device), int(warps), int(cells), int(ring_fwd),
                          int(ring_adj), int(bool(autotune)), _RPREC[radon_precision], int(fd_schedule),
                          {"softmax": 0, "gauss": 1, "wd": 2}[adjoint_weight],
                          {"fp32": 0, "fp64": 1}[image_precision])
        h = ctypes.c_void_p()
        call("swd_engine_create", ctypes.byref(self._sc), ctypes.byref(opts), ctypes.byref(h))
        self._h = h
        inf = EngineInfo()
        call("swd_engine_info", h, ctypes.byref(inf))
        self.info = {k: getattr(inf, k) for k, _ in EngineInfo._fields_}
        self.set_source(survey.source() if source is None else source)
        self._L = L

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().swd_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def npair(self):
        return self.info["npair"]

    def set_source(self, s):
        s = np.ascontiguousarray(np.asarray(s, np.float64).reshape(-1))
        if s.size < self.survey.nt:
            raise ValueError("source wavelet shorter than nt")
        call("swd_engine_set_source", self._h, ptr(s))

    def set_observed(self, cr0_r, cr0_l):
        a, b = _f(cr0_r), _f(cr0_l)
        call("swd_engine_set_observed", self._h, ptr(a), ptr(b))

    def observed_curves(self, vp, vs):
        n = self.npair
        cr, cl = np.zeros((n, self.survey.ns), order="F"), np.zeros((n, self.survey.ns), order="F")
        vp, vs = _f(vp), _f(vs)
        call("swd_engine_observed_curves", self._h, ptr(vp), ptr(vs), ptr(cr), ptr(cl))
        return cr, cl

    def misfit(self, vp, vs):
        ns, n = self.survey.ns, self.npair
        out = {"res_r": np.zeros(ns), "res_l": np.zeros(ns), "cr_pre_r": np.zeros((n, ns), order="F"),
               "cr_pre_l": np.zeros((n, ns), order="F")}
        r = ctypes.c_double()
        vp, vs = _f(vp), _f(vs)
        call("swd_engine_misfit", self._h, ptr(vp), ptr(vs), ptr(out["res_r"]), ptr(out["res_l"]),
             ptr(out["cr_pre_r"]), ptr(out["cr_pre_l"]), ctypes.byref(r))
        out["residual"] = r.value
        return out

    def gradient(self, vp, vs):
        s = self.survey
        shp = (s.nz, s.nx)
        out = {k: np.zeros(shp, order="F") for k in ("g_cl", "g_cm", "g_illum", "dk_vs")}
        out.update(res_r=np.zeros(s.ns), res_l=np.zeros(s.ns), cr_pre_r=np.zeros((self.npair, s.ns), order="F"),
                   cr_pre_l=np.zeros((self.npair, s.ns), order="F"))
        go = GradientOut(*[ptr(out[k]) for k in ("g_cl", "g_cm", "g_illum", "dk_vs", "res_r", "res_l", "cr_pre_r",
                                                  "cr_pre_l")], 0.0)
        vp, vs = _f(vp), _f(vs)
        call("swd_engine_gradient", self._h, ptr(vp), ptr(vs), ctypes.byref(go))
        out["residual"] = go.residual
        return out

    def gradient_device(self, d_vp, d_vs, d_dk=None):
        """Device-resident call: d_vp, d_vs, d_dk are float64 CUDA tensors (nz x nx, column-major data,
        i.e. tensors of shape (nx, nz) contiguous).  Returns the misfit."""
        r = ctypes.c_double()
        call("swd_engine_gradient_device", self._h, ctypes.c_void_p(d_vp.data_ptr()),
             ctypes.c_void_p(d_vs.data_ptr()), ctypes.c_void_p(d_dk.data_ptr() if d_dk is not None else 0),
             ctypes.byref(r))
        return r.value

    def radon_stats(self):
        """Split-BF16 spectra: gathers picked so far and how many were recomputed in FP64 because a
        pick decision fell inside the certification margin."""
        g, r = ctypes.c_uint64(), ctypes.c_uint64()
        call("swd_engine_radon_stats", self._h, ctypes.byref(g), ctypes.byref(r))
        return {"gathers": g.value, "recomputed_fp64": r.value}

    def cancel(self):
        """Cancel the call in flight on this engine (from another thread; returns at once): that
        call raises SwdError with status SWD_ERR_CANCELLED (5); a cancel raised while no call
        runs cancels the next one."""
        call("swd_engine_cancel", self._h)

    def stream(self):
        p = ctypes.c_void_p()
        call("swd_engine_stream", self._h, ctypes.byref(p))
        return p.value

    def shot_sums_device(self, d_vp, d_vs, d_gsum):
        """Shot sums of this engine's shots into d_gsum (3*nz*nx float64 CUDA tensor).
        Returns (right-side misfit sum, count) for a cross-rank mean."""
        rs, rc = ctypes.c_double(), ctypes.c_int()
        call("swd_engine_shot_sums_device", self._h, ctypes.c_void_p(d_vp.data_ptr()),
             ctypes.c_void_p(d_vs.data_ptr()), ctypes.c_void_p(d_gsum.data_ptr()), ctypes.byref(rs),
             ctypes.byref(rc))
        return rs.value, rc.value

    def assemble_device(self, d_gsum, d_dk):
        call("swd_engine_assemble_device", self._h, ctypes.c_void_p(d_gsum.data_ptr()),
             ctypes.c_void_p(d_dk.data_ptr()))

    def set_timing(self, on=True):
        call("swd_engine_set_timing", self._h, int(on))

    def phase_times(self):
        """(forward, spectra, adjoint) milliseconds of the last call (set_timing(True) first)."""
        a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        call("swd_engine_phase_times", self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
        return a.value, b.value, c.value
