"""Dispersion spectrum, picking and SoftMax gradient behind the reference's .m interfaces.

    RTr / RTl / RTrAD / RTlAD   core/RTr.m:2, core/RTl.m:2, core/RTrAD.m:2, core/RTlAD.m:2
    LHDispPick                  core/LHDispPick.m:2 (pickFDC1, core/pickFDC1.m:1)
    ADWDgrad_1                  core/ADWDgrad_1.m:1
    ADWDgrad_norm               core/ADWDgrad_norm.m:1
    ADWDgradlimband             core/ADWDgradlimband.m:1
    weight_data_muti3           core/weight_data_muti3.m:1 (the WD adjoint source)
    norm_trace                  core/norm_trace.m:1
    LHDispPick_field            fieldexamples/outcrop/core/LHDispPick.m:2 (pickFDCValue.m:1),
                                fieldexamples/QadimahFault/core/LHDispPick.m:2 (mode 1)
    ADWDgrad_1_maxnorm          fieldexamples/outcrop/core/ADWDgrad_1.m:1

Each call runs on the GPU through libswd.so (FP64, like the reference's MATLAB
code).  Arrays use MATLAB's layout; saveForBackward is a dict with the
reference's field names plus the transform parameters.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import RadonParams, call, ptr


def radon_params(df, dt, vmin, vmax, fmin, fmax, a, b, ds, offset, m, M, dv=1.0) -> RadonParams:
    return RadonParams(float(df), float(dt), float(fmin), float(fmax), float(vmin), float(vmax), float(dv),
                       float(ds), int(a), int(b), int(offset), int(m), int(M), 0)


def sizes(p: RadonParams):
    out = [ctypes.c_int() for _ in range(5)]
    call("swd_radon_sizes", ctypes.byref(p), *[ctypes.byref(o) for o in out])
    return tuple(o.value for o in out)  # np, npair, lf, nf, ccn


def _radon(side, seismo_v1, is_, df, dt, np_, vmin, vmax, fmin, fmax, a, b, ds, offset, m, M, dv, FK=0):
    seis = np.asfortranarray(np.asarray(seismo_v1, np.float64))
    if seis.shape != (int(a), int(b)):
        raise ValueError(f"seismogram is {seis.shape}, expected a x b = {(a, b)}")
    p = radon_params(df, dt, vmin, vmax, fmin, fmax, a, b, ds, offset, m, M, dv)
    if FK == 1:
        # the field drivers' RTrAD/RTlAD filter the gather (as the transform orders it: the left
        # side reversed) before transforming it; the filtered gather goes back into the same
        # columns of a copy, in the same order, so that swd_radon reads exactly it
        n = ctypes.c_int()
        pos = np.zeros(int(offset) + 1, np.int32)
        nv0 = sizes(p)[0]
        call("swd_radon", ctypes.byref(p), side, int(is_), ptr(seis), ptr(np.zeros((nv0, sizes(p)[1]), order="F")),
             None, None, ctypes.byref(n), ptr(pos))
        cols = np.sort(pos[: n.value]) - 1
        if side == 1:
            cols = cols[::-1]
        seis = seis.copy(order="F")
        seis[:, cols] = fk_filter(seis[:, cols], dt, ds)
    nv, npair, lf, nf, ccn = sizes(p)
    if np_ is not None and int(np_) != nv:
        raise ValueError(f"np={np_} but the velocity axis has {nv} entries")
    ml = np.zeros((nv, npair), order="F")
    raw = np.zeros((nv, npair), order="F")
    mm = np.zeros((nv, nf), np.complex128, order="F")
    n = ctypes.c_int()
    pos = np.zeros(int(offset) + 1, np.int32)
    call("swd_radon", ctypes.byref(p), side, int(is_), ptr(seis), ptr(ml), ptr(raw),
         mm.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(n), ptr(pos))
    pos = pos[: n.value].astype(np.float64)
    v = float(vmin) + float(dv) * np.arange(nv)
    x = (int(m) + np.arange(n.value)) * float(ds)
    save = {"mm": mm, "ll0": 1j * (2 * np.pi * float(df)) * np.outer(1.0 / v, x), "lf": lf, "nf": nf, "ccn": ccn,
            ("mlr" if side == 0 else "mll"): raw, ("uxtposr" if side == 0 else "uxtposl"): pos, "params": p}
    return ml, n.value, save


def RTrAD(seismo_v1, is_, df, dt, np_, vmin, vmax, fmin, fmax, a, b, ds, offset, m, M, dv=1.0, FK=0):
    """[ml,dataLen,saveForBackward]=RTrAD(...) (core/RTrAD.m:2); FK=1 f-k filters the gather first, as
    fieldexamples/QadimahFault/core/RTrAD.m:14-16 does."""
    return _radon(0, seismo_v1, is_, df, dt, np_, vmin, vmax, fmin, fmax, a, b, ds, offset, m, M, dv, FK)


def RTlAD(seismo_v1, is_, df, dt, np_, vmin, vmax, fmin, fmax, a, b, ds, offset, m, M, dv=1.0, FK=0):
    """[ml,dataLen,saveForBackward]=RTlAD(...) (core/RTlAD.m:2); FK=1 f-k filters the gather first, as
    fieldexamples/QadimahFault/core/RTlAD.m:15-17 does."""
    return _radon(1, seismo_v1, is_, df, dt, np_, vmin, vmax, fmin, fmax, a, b, ds, offset, m, M, dv, FK)


def RTr(seismo_v1, is_, df, dt, np_, vmin, vmax, fmin, fmax, a, b, ds, offset, m, M, dv=1.0, FK=0):
    """[ml,dataLen]=RTr(...) (core/RTr.m:2); FK as in RTrAD."""
    ml, n, _ = RTrAD(seismo_v1, is_, df, dt, np_, vmin, vmax, fmin, fmax, a, b, ds, offset, m, M, dv, FK)
    return ml, n


def RTl(seismo_v1, is_, df, dt, np_, vmin, vmax, fmin, fmax, a, b, ds, offset, m, M, dv=1.0, FK=0):
    """[ml,dataLen]=RTl(...) (core/RTl.m:2); FK as in RTlAD."""
    ml, n, _ = RTlAD(seismo_v1, is_, df, dt, np_, vmin, vmax, fmin, fmax, a, b, ds, offset, m, M, dv, FK)
    return ml, n


def LHDispPick(ml, vmin, cr_0, method=1, ini=10):
    """[res,cr_pre]=LHDispPick(ml,vmin,cr_0,method,ini) (core/LHDispPick.m:2)."""
    ml = np.asfortranarray(np.asarray(ml, np.float64))
    nv, npair = ml.shape
    cr0 = np.ascontiguousarray(np.broadcast_to(np.asarray(cr_0, np.float64).reshape(-1), (npair,)))
    cr = np.zeros(npair)
    res = ctypes.c_double()
    call("swd_pick", ptr(ml), nv, npair, float(vmin), ptr(cr0), int(method), int(ini), ctypes.byref(res), ptr(cr))
    return res.value, cr


def LHDispPick_field(ml, vmin, cr_0, method, saveForBackward, variant=1):
    """[res,cr_pre]=LHDispPick(ml,vmin,cr_0,method,saveForBackward) of the field-data drivers:
    variant 1 fieldexamples/outcrop/core/LHDispPick.m:2 (pickFDCValue seeded at the global maximum
    of saveForBackward.mlr / .mll, misfit over rows 15..end-15), variant 2
    fieldexamples/QadimahFault/core/LHDispPick.m:2 (its mode 1: pickFDC1 from that column, misfit
    over rows 50..end-30)."""
    ml = np.asfortranarray(np.asarray(ml, np.float64))
    nv, npair = ml.shape
    sv = saveForBackward
    raw = np.asfortranarray(np.asarray(sv["mlr"] if "uxtposr" in sv else sv["mll"], np.float64))
    if raw.shape != ml.shape:
        raise ValueError("saveForBackward's spectrum does not match ml")
    cr0 = np.ascontiguousarray(np.broadcast_to(np.asarray(cr_0, np.float64).reshape(-1), (npair,)))
    cr = np.zeros(npair)
    res = ctypes.c_double()
    call("swd_pick_field", ptr(ml), ptr(raw), nv, npair, float(vmin), ptr(cr0), int(method), int(variant),
         ctypes.byref(res), ptr(cr))
    return res.value, cr


def fk_filter(d, dt, dx):
    """[dfk]=fk_filter(d,dt,dx) (core/fk_filter.m:1): the f-k dip filter of the field drivers."""
    d = np.asfortranarray(np.asarray(d, np.float64))
    if d.ndim != 2:
        raise ValueError("fk_filter takes a 2-D gather (time x traces)")
    out = np.zeros(d.shape, order="F")
    call("swd_fk_filter", ptr(d), d.shape[0], d.shape[1], float(dt), float(dx), ptr(out))
    return out


def norm_trace(data_in):
    """data_out = norm_trace(data_in) (core/norm_trace.m:1): every trace over its largest magnitude."""
    d = np.asfortranarray(np.asarray(data_in, np.float64))
    out = np.zeros(d.shape, order="F")
    call("swd_norm_trace", ptr(d), d.shape[0], d.shape[1], ptr(out))
    return out


def ADWDgrad_1_maxnorm(nt, ng, ns, npair, is_, w, m, M, SoftArgNorm, grad_outputr, grad_outputl, space_M,
                       saveForBackwardr, saveForBackwardl):
    """[a_data_res]=ADWDgrad_1(...) of fieldexamples/outcrop/core/ADWDgrad_1.m:1: the adjoint source
    divided by its largest magnitude (:79)."""
    return _adwdgrad(3, nt, ng, ns, npair, is_, w, m, M, SoftArgNorm, grad_outputr, grad_outputl, space_M,
                     saveForBackwardr, saveForBackwardl)


def ADWDgrad_norm(nt, ng, ns, npair, is_, w, m, M, SoftArgNorm, grad_outputr, grad_outputl, space_M,
                  saveForBackwardr, saveForBackwardl):
    """[a_data_res]=ADWDgrad_norm(...) (core/ADWDgrad_norm.m:1): ADWDgrad_1 with normpdf weights
    around the picks; the saveForBackward dicts carry cr_r / cr_l = cr_pre - vmin (SWD.m:178,184)."""
    return _adwdgrad(True, nt, ng, ns, npair, is_, w, m, M, SoftArgNorm, grad_outputr, grad_outputl, space_M,
                     saveForBackwardr, saveForBackwardl)


def ADWDgradlimband(nt, ng, ns, npair, is_, w, m, M, SoftArgNorm, grad_outputr, grad_outputl, space_M,
                    saveForBackwardr, saveForBackwardl):
    """[a_data_res]=ADWDgradlimband(...) (core/ADWDgradlimband.m:1): power-normalised weights
    mlr.^SoftArgNorm and a 25-bin linear ramp below lf and above nf of the adjoint spectrum."""
    return _adwdgrad(2, nt, ng, ns, npair, is_, w, m, M, SoftArgNorm, grad_outputr, grad_outputl, space_M,
                     saveForBackwardr, saveForBackwardl)


def ADWDgrad_1(nt, ng, ns, npair, is_, w, m, M, SoftArgNorm, grad_outputr, grad_outputl, space_M,
               saveForBackwardr, saveForBackwardl):
    """[a_data_res]=ADWDgrad_1(...) (core/ADWDgrad_1.m:1)."""
    return _adwdgrad(False, nt, ng, ns, npair, is_, w, m, M, SoftArgNorm, grad_outputr, grad_outputl, space_M,
                     saveForBackwardr, saveForBackwardl)


def _adwdgrad(gauss, nt, ng, ns, npair, is_, w, m, M, SoftArgNorm, grad_outputr, grad_outputl, space_M,
              saveForBackwardr, saveForBackwardl):
    sr = saveForBackwardr if isinstance(saveForBackwardr, dict) else None
    sl = saveForBackwardl if isinstance(saveForBackwardl, dict) else None
    p = (sr or sl)["params"]
    if int(p.nt) != int(nt) or int(p.ng) != int(ng) or int(p.m) != int(m) or int(p.M) != int(M):
        raise ValueError("nt/ng/m/M differ from the ones the spectrum was computed with")
    a = np.zeros((int(nt), int(ng)), order="F")
    dp = ctypes.POINTER(ctypes.c_double)

    def side(s, go, rawkey):
        if s is None:
            return None, None, None
        mm = np.asfortranarray(s["mm"].astype(np.complex128))
        raw = np.asfortranarray(np.asarray(s[rawkey], np.float64))
        g = np.ascontiguousarray(np.asarray(go, np.float64).reshape(-1)[: int(npair)])
        return mm, raw, g

    mmr, rawr, gr = side(sr, grad_outputr, "mlr")
    mml, rawl, gl = side(sl, grad_outputl, "mll")
    spm = None if space_M is None else np.asfortranarray(np.asarray(space_M, np.float64))
    cp = lambda x: None if x is None else x.ctypes.data_as(dp)
    if gauss == 3:
        call("swd_adwdgrad_maxnorm", ctypes.byref(p), int(ns), int(is_), int(w), float(SoftArgNorm), cp(gr), cp(gl),
             cp(spm), cp(mmr), cp(rawr), cp(mml), cp(rawl), ptr(a))
    elif gauss == 2:
        call("swd_adwdgrad_limband", ctypes.byref(p), int(ns), int(is_), int(w), float(SoftArgNorm), cp(gr), cp(gl),
             cp(spm), cp(mmr), cp(rawr), cp(mml), cp(rawl), ptr(a))
    elif gauss:
        def picks(sv, key):
            return None if sv is None else np.ascontiguousarray(np.asarray(sv[key], np.float64).reshape(-1))
        crr, crl = picks(sr, "cr_r"), picks(sl, "cr_l")
        call("swd_adwdgrad_norm", ctypes.byref(p), int(ns), int(is_), int(w), float(SoftArgNorm), cp(gr), cp(gl),
             cp(spm), cp(mmr), cp(rawr), cp(crr), cp(mml), cp(rawl), cp(crl), ptr(a))
    else:
        call("swd_adwdgrad", ctypes.byref(p), int(ns), int(is_), int(w), float(SoftArgNorm), cp(gr), cp(gl),
             cp(spm), cp(mmr), cp(rawr), cp(mml), cp(rawl), ptr(a))
    return a


def weight_data_muti3(seismo_v_d, seismo_v, is_, dt, df, offset, dg, F1, w, M, m, ns, refsx, win, fmin, fmax,
                      cr_0, cr_0l, cr_pre_r, cr_pre_l, ind):
    """[seismo_v_d1]=weight_data_muti3(...) (core/weight_data_muti3.m:1), the WD adjoint source
    that SWD.m:188 offers: F1=0 filters the predicted data seismo_v, F1=1 the observed data
    seismo_v_d (the other may be None).  Returns seismo_v_d1 (nt x ng)."""
    src = seismo_v_d if int(F1) == 1 else seismo_v
    if src is None:
        raise ValueError("F1=1 needs seismo_v_d, F1=0 needs seismo_v")
    src = np.asfortranarray(np.asarray(src, np.float64))
    if src.ndim != 2:
        raise ValueError("seismograms must be nt x ng")
    nt, ng = src.shape
    other = seismo_v if int(F1) == 1 else seismo_v_d
    if other is not None and np.shape(other)[:2] != (nt, ng):
        raise ValueError("seismo_v_d and seismo_v differ in size")
    refsx = np.ascontiguousarray(np.asarray(refsx, np.float64).reshape(-1))
    if refsx.size < int(ns):
        raise ValueError(f"refsx has {refsx.size} entries, ns is {ns}")
    npair = int(np.floor((fmax - fmin) / df + 1))
    dp = ctypes.POINTER(ctypes.c_double)

    def picks(a):
        if a is None:
            return None
        a = np.ascontiguousarray(np.asarray(a, np.float64).reshape(-1))
        if a.size != npair:
            raise ValueError(f"picks have {a.size} entries, linspace(fmin, fmax, ...) has {npair}")
        return a
    crs = [picks(a) for a in (cr_0, cr_0l, cr_pre_r, cr_pre_l)]
    out = np.zeros((nt, ng), order="F")
    cp = lambda x: None if x is None else x.ctypes.data_as(dp)
    call("swd_wd_residual", nt, ng, cp(src) if int(F1) == 1 else None, cp(src) if int(F1) == 0 else None, int(is_),
         float(dt), float(df), int(offset), float(dg), int(F1), int(w), float(M), int(m), int(ns),
         refsx.ctypes.data_as(dp), int(win), float(fmin), float(fmax), *[cp(c) for c in crs], int(ind), ptr(out))
    return out
