"""FD forward modelling and adjoint imaging behind the reference's own interfaces.

MEX level (same arguments and outputs as the reference's MEX files):
    eigen_staggerfd_single / eigen_staggerfd_double
        core/eigen_staggerfd_single.cpp:68-383 (double: binary-only, interface at
        core/staggerfd_eigend.m:139)
    eigen_e2drtm_single / eigen_e2drtm_double
        core/eigen_e2drtm_single.cpp:67-296 (double: core/e2drtm_eigend.m:122)
.m level (same signatures as the wrappers):
    staggerfd_eigen / staggerfd_eigend   core/staggerfd_eigen.m:2, core/staggerfd_eigend.m:2
    e2drtm_eigen / e2drtm_eigend         core/e2drtm_eigen.m:8, core/e2drtm_eigend.m:8

All arrays follow MATLAB's layout (column-major numpy arrays); every
computation runs in libswd.so on the GPU.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import call, lib, ptr

_SRC = {"p": 1, "s": 2, "s1": 3, "z": 4, "w": 5}  # core/staggerfd_eigen.m:126-136


def _f(a, dt):
    return np.asfortranarray(np.asarray(a, dt))


class _FdJob(ctypes.Structure):
    """swd_staggerfd_job of include/swd.h."""
    _fields_ = [("iv", ctypes.c_void_p), ("n_iv", ctypes.c_int)] + \
               [(k, ctypes.c_void_p) for k in ("temp", "ca", "cl", "cm", "cm1", "b", "b1", "s", "seismo_u",
                                                "seismo_w", "fux", "fuz", "bwx", "bwz")]


class KeptWavefields:
    """The strain snapshots of a forward batch, kept on the device for eigen_e2drtm_single_batch
    (swd_staggerfd_single_batch_keep); released when this object goes."""

    def __init__(self, handle, n_jobs):
        self.handle, self.n_jobs = handle, n_jobs

    def __del__(self):
        if self.handle:
            lib().swd_fd_batch_free(self.handle)
            self.handle = None


def eigen_staggerfd_single_batch(jobs, want_wf=False, keep=False):
    """Several eigen_staggerfd_single calls, on grids of any sizes, advanced together by one launch per
    time step; it has no counterpart in the reference (one MEX call per shot and model).  jobs: a
    list of (iv, temp, ca, cl, cm, cm1, b, b1, s) as for eigen_staggerfd_single.  Returns
    [(seismo_u, seismo_w, www or None)], bit for bit those of the separate calls; with keep, also
    a KeptWavefields holding every job's snapshots on the device for eigen_e2drtm_single_batch."""
    alive, outs = [], []
    arr = (_FdJob * len(jobs))()
    for k, (iv, temp, ca, cl, cm, cm1, b, b1, s) in enumerate(jobs):
        iv = np.ascontiguousarray(np.asarray(iv, np.float32).reshape(-1))
        nt, ng, nz, nx, ntwf = int(iv[0]), int(iv[4]), int(iv[13]), int(iv[14]), int(iv[12])
        mats = [_f(a, np.float32) for a in (temp, ca, cl, cm, cm1, b, b1)]
        s = np.ascontiguousarray(np.asarray(s, np.float32).reshape(-1))
        if s.size < nt:
            raise ValueError(f"job {k}: source wavelet has {s.size} samples, nt={nt}")
        su = np.zeros((nt, ng), np.float32, order="F")
        sw = np.zeros((nt, ng), np.float32, order="F")
        wf = ({f: np.zeros((nz, nx, nt // max(ntwf, 1)), np.float32, order="F") for f in ("fux", "fuz", "bwx", "bwz")}
              if want_wf else None)
        alive += [iv, s, *mats]
        outs.append((su, sw, wf))
        w = [wf[f].ctypes.data if wf else None for f in ("fux", "fuz", "bwx", "bwz")]
        arr[k] = _FdJob(iv.ctypes.data, iv.size, *[m.ctypes.data for m in mats], s.ctypes.data, su.ctypes.data,
                        sw.ctypes.data, *w)
    if not keep:
        call("swd_staggerfd_single_batch", len(jobs), ctypes.cast(arr, ctypes.c_void_p))
        return outs
    h = ctypes.c_void_p()
    call("swd_staggerfd_single_batch_keep", len(jobs), ctypes.cast(arr, ctypes.c_void_p), ctypes.byref(h))
    return outs, KeptWavefields(h.value, len(jobs))


class _AdjJob(ctypes.Structure):
    """swd_e2drtm_job of include/swd.h."""
    _fields_ = [("iv", ctypes.c_void_p), ("n_iv", ctypes.c_int)] + \
               [(k, ctypes.c_void_p) for k in ("temp", "ca", "cl", "cm", "cm1", "b", "b1", "seismo_w", "fux", "fuz",
                                                "bwx", "bwz", "cl_img", "cm_img", "illum_div")]


def eigen_e2drtm_single_batch(jobs, kept=None):
    """Several eigen_e2drtm_single calls, on grids of any sizes, advanced together by one launch per
    time step (no counterpart in the reference).  jobs: a list of (iv, temp, ca, cl, cm, cm1, b, b1,
    seismo_w, fux, fuz, bwx, bwz) as for eigen_e2drtm_single.  Returns [(cl_img, cm_img, illum_div)],
    FP32 as the single MEX, bit for bit those of the separate calls.  kept: the KeptWavefields of
    the forward batch of the same jobs, whose device snapshots job k then reads in place of its
    fux..bwz (which may be None)."""
    if kept is not None and kept.n_jobs != len(jobs):
        raise ValueError(f"the kept forward batch has {kept.n_jobs} jobs, this batch {len(jobs)}")
    keep, outs = [], []
    arr = (_AdjJob * len(jobs))()
    for k, job in enumerate(jobs):
        iv = np.ascontiguousarray(np.asarray(job[0], np.float32).reshape(-1))
        nz, nx = int(iv[11]), int(iv[12])
        ins = [None if (a is None and kept is not None and i >= 10) else _f(a, np.float32)
               for i, a in enumerate(job[1:], 1)]
        img = [np.zeros((nz, nx), np.float32, order="F") for _ in range(3)]
        keep += [iv, *ins]
        outs.append(tuple(img))
        arr[k] = _AdjJob(iv.ctypes.data, iv.size, *[None if a is None else a.ctypes.data for a in ins],
                         *[o.ctypes.data for o in img])
    if kept is None:
        call("swd_e2drtm_single_batch", len(jobs), ctypes.cast(arr, ctypes.c_void_p))
    else:
        call("swd_e2drtm_single_batch_kept", len(jobs), ctypes.cast(arr, ctypes.c_void_p),
             ctypes.c_void_p(kept.handle))
    return outs


def _mex_fwd(fn, dt, iv, temp, ca, cl, cm, cm1, b, b1, s, want_wf=True):
    iv = np.ascontiguousarray(np.asarray(iv, dt).reshape(-1))
    nt, ng, nz, nx, ntwf = int(iv[0]), int(iv[4]), int(iv[13]), int(iv[14]), int(iv[12])
    args = [_f(a, dt) for a in (temp, ca, cl, cm, cm1, b, b1)]
    s = np.ascontiguousarray(np.asarray(s, dt).reshape(-1))
    if s.size < nt:
        raise ValueError(f"source wavelet has {s.size} samples, nt={nt}")
    su = np.zeros((nt, ng), dt, order="F")
    sw = np.zeros((nt, ng), dt, order="F")
    nrec = nt // max(ntwf, 1)
    wf = {k: np.zeros((nz, nx, nrec), dt, order="F") for k in ("fux", "fuz", "bwx", "bwz")} if want_wf else None
    w = [ptr(wf[k]) if wf else None for k in ("fux", "fuz", "bwx", "bwz")]
    call(fn, ptr(iv), iv.size, *[ptr(a) for a in args], ptr(s), ptr(su), ptr(sw), *w)
    return su, sw, wf


def eigen_staggerfd_single(iv, temp, ca, cl, cm, cm1, b, b1, s, want_wf=True):
    """[seismo_u, seismo_w, www] = eigen_staggerfd_single(iv,temp,ca,cl,cm,cm1,b,b1,s)."""
    return _mex_fwd("swd_staggerfd_single", np.float32, iv, temp, ca, cl, cm, cm1, b, b1, s, want_wf)


def eigen_staggerfd_double(iv, temp, ca, cl, cm, cm1, b, b1, s, want_wf=True):
    """[seismo_u, seismo_w, www] = eigen_staggerfd_double(...) in FP64."""
    return _mex_fwd("swd_staggerfd_double", np.float64, iv, temp, ca, cl, cm, cm1, b, b1, s, want_wf)


def _mex_adj(fn, dt, out_dt, iv, temp, ca, cl, cm, cm1, b, b1, seismo_w, fux, fuz, bwx, bwz):
    iv = np.ascontiguousarray(np.asarray(iv, dt).reshape(-1))
    nz, nx = int(iv[11]), int(iv[12])
    args = [_f(a, dt) for a in (temp, ca, cl, cm, cm1, b, b1, seismo_w, fux, fuz, bwx, bwz)]
    outs = [np.zeros((nz, nx), out_dt, order="F") for _ in range(3)]
    call(fn, ptr(iv), iv.size, *[ptr(a) for a in args], *[ptr(o) for o in outs])
    return tuple(outs)


def eigen_e2drtm_single(iv, temp, ca, cl, cm, cm1, b, b1, seismo_w, fux, fuz, bwx, bwz, fp64_out=False):
    """[cl_img, cm_img, illum_div] = eigen_e2drtm_single(...): single images accumulated in FP32 as
    the reference MEX does; fp64_out=True accumulates in FP64 and returns double images."""
    if fp64_out:
        return _mex_adj("swd_e2drtm_single_f64out", np.float32, np.float64, iv, temp, ca, cl, cm, cm1, b, b1,
                        seismo_w, fux, fuz, bwx, bwz)
    return _mex_adj("swd_e2drtm_single", np.float32, np.float32, iv, temp, ca, cl, cm, cm1, b, b1, seismo_w, fux,
                    fuz, bwx, bwz)


def eigen_e2drtm_double(iv, temp, ca, cl, cm, cm1, b, b1, seismo_w, fux, fuz, bwx, bwz):
    """[cl_img, cm_img, illum_div] = eigen_e2drtm_double(...)."""
    return _mex_adj("swd_e2drtm_double", np.float64, np.float64, iv, temp, ca, cl, cm, cm1, b, b1, seismo_w, fux, fuz,
                    bwx, bwz)


def prep_model(nbc, dtx, dx, dt, vp, vs, isfs=1, fd_order=22, single=True):
    """Padded FD inputs built on the GPU as core/staggerfd_eigen.m:37-107 does.

    Returns dict temp, ca, cl, cm, cm1, b, b1 (nzbc x nxbc, column-major) and pad_top.
    """
    vp = _f(vp, np.float64)
    vs = _f(vs, np.float64)
    nz, nx = vs.shape
    if vp.shape != vs.shape:
        raise ValueError("vp and vs must have the same shape")
    pad_top = (fd_order - 20) // 2 + 1
    NZ, NX = nz + pad_top + nbc, nx + 2 * nbc
    dt_ = np.float32 if single else np.float64
    out = {k: np.zeros((NZ, NX), dt_, order="F") for k in ("temp", "ca", "cl", "cm", "cm1", "b", "b1")}
    fn = "swd_prep_model_single" if single else "swd_prep_model_double"
    call(fn, nz, nx, nbc, int(isfs), fd_order, float(dx), float(dt), float(dtx), ptr(vp), ptr(vs),
         *[ptr(out[k]) for k in ("temp", "ca", "cl", "cm", "cm1", "b", "b1")])
    out["pad_top"] = pad_top
    return out


def _geometry(nbc, pad_top, gx, gz):
    gx = np.atleast_1d(np.asarray(gx, np.float64)).reshape(-1)
    gz = np.atleast_1d(np.asarray(gz, np.float64)).reshape(-1)
    if gx.size < 2:
        raise ValueError("need at least two receivers (the wrappers read gx(2)-gx(1))")
    return gx.size, gz[0] + pad_top, gx[0] + nbc, gx[1] - gx[0]


def staggerfd_mex_args(nbc, nt, dtx, dx, dt, sx, sz, gx, gz, vp, vs, isfs, fd_order, source_type, parameter_type,
                       in_wf, single=True, m=None):
    """The MEX arguments (iv, temp, ca, cl, cm, cm1, b, b1) that core/staggerfd_eigen.m:37-138
    builds; m: prep_model's output when the caller already has it (the same for every shot)."""
    if parameter_type != 0:
        raise ValueError("parameter_type=1 reads undefined cl/cm in core/staggerfd_eigen.m:43-45")
    if m is None:
        m = prep_model(nbc, dtx, dx, dt, vp, vs, isfs, fd_order, single)
    nz, nx = np.asarray(vs).shape
    NZ, NX = m["temp"].shape
    ng, gz0, gx0, dg = _geometry(nbc, m["pad_top"], gx, gz)
    iv = [nt, NZ, NX, dtx, ng, float(sz) + m["pad_top"], float(sx) + nbc, gz0, gx0, dg, _SRC[source_type], fd_order,
          in_wf, nz, nx, 3]  # core/staggerfd_eigen.m:138
    return (iv, m["temp"], m["ca"], m["cl"], m["cm"], m["cm1"], m["b"], m["b1"])


def _staggerfd(single, is_, nbc, nt, dtx, dx, dt, sx, sz, gx, gz, s, vp, vs, isfs, fd_order, source_type,
               parameter_type, in_wf):
    args = staggerfd_mex_args(nbc, nt, dtx, dx, dt, sx, sz, gx, gz, vp, vs, isfs, fd_order, source_type,
                              parameter_type, in_wf, single)
    fn = eigen_staggerfd_single if single else eigen_staggerfd_double
    return fn(*args, s)


def staggerfd_eigen(is_, nbc, nt, dtx, dx, dt, sx, sz, gx, gz, s, vp, vs, isfs=1, fd_order=22, source_type="w",
                    parameter_type=0, in_wf=5):
    """[seismo_u,seismo_w,www]=staggerfd_eigen(...) (core/staggerfd_eigen.m:2)."""
    return _staggerfd(True, is_, nbc, nt, dtx, dx, dt, sx, sz, gx, gz, s, vp, vs, isfs, fd_order, source_type,
                      parameter_type, in_wf)


def staggerfd_eigend(is_, nbc, nt, dtx, dx, dt, sx, sz, gx, gz, s, vp, vs, isfs=1, fd_order=22, source_type="w",
                     parameter_type=0, in_wf=5):
    """[seismo_u,seismo_w,www]=staggerfd_eigend(...) (core/staggerfd_eigend.m:2), FP64."""
    return _staggerfd(False, is_, nbc, nt, dtx, dx, dt, sx, sz, gx, gz, s, vp, vs, isfs, fd_order, source_type,
                      parameter_type, in_wf)


def staggerfd_eigen_field(is_, nbc, nt, dtx, dx, dt, sx, sz, gx, gz, s, vp, vs, isfs, fsz, fd_order, source_type,
                          parameter_type, dt_wf=None, nt_wf=None):
    """[seismo_u,seismo_w,www]=staggerfd_eigen(...) of the QadimahFault driver
    (fieldexamples/QadimahFault/core/staggerfd_eigen.m:2, function staggerfd8): core's wrapper with
    the snapshot interval given as a time, in_wf = dt_wf/dt (:157; dt_wf = dt when omitted,
    :37-40).  fsz and nt_wf are accepted and unused, as there."""
    in_wf = (dt if dt_wf is None else dt_wf) / dt  # goes to the single input vector, as there
    return _staggerfd(True, is_, nbc, nt, dtx, dx, dt, sx, sz, gx, gz, s, vp, vs, isfs, fd_order, source_type,
                      parameter_type, in_wf)


def e2drtm_mex_args(wavefield_gradient, seismo_w, nbc, nt, dtx, dx, dt, gx, gz, vp, vs, isfs, fd_order,
                    parameter_type, in_wf, single=True, m=None):
    """The MEX arguments (iv, temp, ca, cl, cm, cm1, b, b1, seismo_w, fux, fuz, bwx, bwz) that
    core/e2drtm_eigen.m:44-122 builds; m as in staggerfd_mex_args."""
    if parameter_type != 0:
        raise ValueError("parameter_type=1 reads undefined cl/cm in core/e2drtm_eigen.m:49-51")
    if m is None:
        m = prep_model(nbc, dtx, dx, dt, vp, vs, isfs, fd_order, single)
    nz, nx = np.asarray(vs).shape
    NZ, NX = m["temp"].shape
    ng, gz0, gx0, dg = _geometry(nbc, m["pad_top"], gx, gz)
    iv = [nt, NZ, NX, dtx, ng, nbc, gz0, gx0, dg, fd_order, in_wf, nz, nx, dt]  # core/e2drtm_eigen.m:121
    wg = wavefield_gradient
    return (iv, m["temp"], m["ca"], m["cl"], m["cm"], m["cm1"], m["b"], m["b1"], seismo_w, wg["fux"], wg["fuz"],
            wg["bwx"], wg["bwz"])


def _e2drtm(single, wavefield_gradient, seismo_w, is_, nbc, nt, dtx, dx, dt, gx, gz, s, vp, vs, isfs, fd_order,
            parameter_type, in_wf, fp64_out=False):
    args = e2drtm_mex_args(wavefield_gradient, seismo_w, nbc, nt, dtx, dx, dt, gx, gz, vp, vs, isfs, fd_order,
                           parameter_type, in_wf, single)
    if single:
        return eigen_e2drtm_single(*args, fp64_out=fp64_out)
    return eigen_e2drtm_double(*args)


def e2drtm_eigen(wavefield_gradient, seismo_w, is_, nbc, nt, dtx, dx, dt, gx, gz, s, vp, vs, isfs=1, fd_order=22,
                 parameter_type=0, in_wf=5, fp64_out=False):
    """[cl_img,cm_img,illum_div]=e2drtm_eigen(...) (core/e2drtm_eigen.m:8)."""
    return _e2drtm(True, wavefield_gradient, seismo_w, is_, nbc, nt, dtx, dx, dt, gx, gz, s, vp, vs, isfs, fd_order,
                   parameter_type, in_wf, fp64_out)


def e2drtm_eigen_field(wavefield_gradient, seismo_w, is_, nbc, nt, dtx, dx, dt, gx, gz, s, vp, vs, isfs, fsz, fd_order,
                       parameter_type, dt_wf=None, fp64_out=False):
    """[cl_img,cm_img,illum_div]=e2drtm_eigen(...) of the QadimahFault driver
    (fieldexamples/QadimahFault/core/e2drtm_eigen.m:8): core's wrapper with in_wf = dt_wf/dt (:147;
    dt_wf = dt when omitted, :43-45).  fsz only enters statements without effect there (:85-87, :94)."""
    in_wf = (dt if dt_wf is None else dt_wf) / dt
    return _e2drtm(True, wavefield_gradient, seismo_w, is_, nbc, nt, dtx, dx, dt, gx, gz, s, vp, vs, isfs, fd_order,
                   parameter_type, in_wf, fp64_out)


def e2drtm_eigend(wavefield_gradient, seismo_w, is_, nbc, nt, dtx, dx, dt, gx, gz, s, vp, vs, isfs=1, fd_order=22,
                  parameter_type=0, in_wf=5):
    """[cl_img,cm_img,illum_div]=e2drtm_eigend(...) (core/e2drtm_eigend.m:8), FP64."""
    return _e2drtm(False, wavefield_gradient, seismo_w, is_, nbc, nt, dtx, dx, dt, gx, gz, s, vp, vs, isfs, fd_order,
                   parameter_type, in_wf)
