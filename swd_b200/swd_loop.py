"""The shot loops of SWD.m / SWD_single.m on the MEX-convention entry points.

This is what the reference's driver runs once the MEX shims stand in for its MEX files:
one shot per call, as the body of its parfor (SWD.m:171-201), with the spectra, picks and
SoftMax adjoint sources of the .m functions (RTrAD/RTlAD, LHDispPick, ADWDgrad_1).

    single=True   SWD_single.m: FP32 FD (eigen_staggerfd_single / eigen_e2drtm_single), the
                  adjoint source cast to single (SWD_single.m:193)
    single=False  SWD.m: FP64 FD (the _double MEX pair), all in double

    field=1       the field-data flow of fieldexamples/outcrop/outcrop.m:168-196: each predicted
                  gather trace-normalised (norm_trace), picks seeded at the spectrum's global
                  maximum with the misfit over rows 15..end-15 (that directory's LHDispPick /
                  pickFDCValue), the adjoint source divided by its largest magnitude (its
                  ADWDgrad_1.m:79); the observed curves are the caller's (manual picks,
                  outcrop.m:137-160).  The outcrop driver runs it with single=False (its wrappers
                  call the _double MEX, staggerfd_eigen.m:139-141 there).
    field=2       the same with fieldexamples/QadimahFault's picker (pickFDC1 from the column
                  of the global maximum, misfit over rows 50..end-30).

The batched engine (swd_b200.engine) computes the same gradient in one pipeline; this loop
is the per-shot path and the full-FP64 path the engine's precision is measured against.
Images are accumulated in FP64 in both modes.
"""
from __future__ import annotations

import math

import numpy as np

from .fd import e2drtm_eigen, e2drtm_eigend, staggerfd_eigen, staggerfd_eigend
from .spectrum import ADWDgrad_1, ADWDgrad_1_maxnorm, LHDispPick, LHDispPick_field, RTlAD, RTrAD, norm_trace


def _mround(x):
    return int(math.floor(x + 0.5)) if x >= 0 else -int(math.floor(-x + 0.5))


def has_right(is_, ns, m, M, w):
    """ADWDgrad_1.m:13 / SWD.m:175."""
    return is_ <= ns - math.floor(m / M) - _mround(w / M)


def has_left(is_, m, M, w):
    """ADWDgrad_1.m:46 / SWD.m:181."""
    return is_ >= _mround(w / M) + math.floor(m / M) + 1


def smooth2a(a, nr, nc):
    """smooth2a(A, Nr, Nc) (core/smooth2a.m:52-76): mean over the (2Nr+1) x (2Nc+1) window
    clipped to the grid; NaNs are left out of sums and counts and stay NaN."""
    a = np.asarray(a, np.float64)
    nz, nx = a.shape
    ok = ~np.isnan(a)
    v = np.where(ok, a, 0.0)
    s = np.zeros_like(v)
    n = np.zeros_like(v)
    for dz in range(-nr, nr + 1):
        for dx in range(-nc, nc + 1):
            z0, z1 = max(0, -dz), min(nz, nz - dz)
            x0, x1 = max(0, -dx), min(nx, nx - dx)
            s[z0:z1, x0:x1] += v[z0 + dz:z1 + dz, x0 + dx:x1 + dx]
            n[z0:z1, x0:x1] += ok[z0 + dz:z1 + dz, x0 + dx:x1 + dx]
    out = s / n
    out[~ok] = np.nan
    return out


def _seismogram(s, is_, vs, single, want_wf=True):
    fd = staggerfd_eigen if single else staggerfd_eigend
    su, sw, www = fd(is_, s.nbc, s.nt, s.dtx, s.dx, s.dt, int(s.sx[is_ - 1]), 1, s.gx, np.ones(s.ng), s.source(),
                     s.vp_ratio * vs, vs, s.isfs, s.fd_order, s.source_type, 0, s.nt_wf)
    return sw, www


def spectra(s, seismo, is_, FK=0):
    """RTrAD / RTlAD of one shot's vertical-component record for the sides it has (SWD.m:174-185);
    FK=1 f-k filters the gathers first (the field drivers' option)."""
    shot_no = int(s.shot_no[is_ - 1]) if s.shot_no is not None else is_
    ns = s.ns_total or s.ns
    args = (shot_no, s.df, s.dt, s.np_vel, s.vmin, s.vmax, s.fmin, s.fmax, s.nt, s.ng, s.ds, s.offset, s.m, s.M,
            s.dv)
    out = {}
    if has_right(shot_no, ns, s.m, s.M, s.w):
        out["r"] = RTrAD(np.asarray(seismo, np.float64), *args, FK=FK)
    if has_left(shot_no, s.m, s.M, s.w):
        out["l"] = RTlAD(np.asarray(seismo, np.float64), *args, FK=FK)
    return out


def _shot_adjoint_source(s, is_, sw, cr0_r, cr0_l, single, field, FK):
    """SWD.m:174-193 for shot is_ from its predicted gather sw: spectra, picks, misfits and the
    adjoint source (FP32 on the single path, SWD_single.m:193)."""
    if field:
        # outcrop.m:174; on single data MATLAB divides in single (the FP64 quotient rounded to
        # FP32 is that same single quotient)
        sw = norm_trace(sw).astype(np.float32) if single else norm_trace(sw)
    sp = spectra(s, sw, is_, FK)
    npair = s.npair
    shot_no = int(s.shot_no[is_ - 1]) if s.shot_no is not None else is_
    ns = s.ns_total or s.ns
    out = {"seismo_w": sw, "res_r": np.nan, "res_l": np.nan, "crp_r": np.ones(npair), "crp_l": np.ones(npair)}
    def pick(sd, cr0):
        if field:
            return LHDispPick_field(sd[0], s.vmin, cr0, 1, sd[2], variant=field)
        return LHDispPick(sd[0], s.vmin, cr0, 1, s.ini)

    if "r" in sp:
        out["ml_r"] = sp["r"][0]
        out["res_r"], out["crp_r"] = pick(sp["r"], cr0_r[:, is_ - 1])
    if "l" in sp:
        out["ml_l"] = sp["l"][0]
        out["res_l"], out["crp_l"] = pick(sp["l"], cr0_l[:, is_ - 1])
    gr = out["crp_r"] - cr0_r[:, is_ - 1]  # SWD.m:186-187
    gl = out["crp_l"] - cr0_l[:, is_ - 1]
    space = np.repeat(np.arange(1.0, s.np_vel + 1)[:, None], npair, 1)  # SWD.m:133-136
    adj = ADWDgrad_1_maxnorm if field else ADWDgrad_1
    a = adj(s.nt, s.ng, ns, npair, shot_no, s.w, s.m, s.M, s.soft_arg_norm, gr, gl, space,
            sp["r"][2] if "r" in sp else None, sp["l"][2] if "l" in sp else None)
    return out, (a.astype(np.float32) if single else a)


def shot_gradient(s, is_, vs, cr0_r, cr0_l, single=True, field=0, FK=0):
    """SWD.m:172-193 for shot is_ (1-based in s): images cl, cm, illum plus picks and misfits
    (field 1 / 2: the field-data flow, see the module docstring; FK=1: the gathers f-k filtered
    before the transform, QademahSWD3.m:119)."""
    sw, www = _seismogram(s, is_, vs, single)
    out, a = _shot_adjoint_source(s, is_, sw, cr0_r, cr0_l, single, field, FK)
    if single:
        cl, cm, il = e2drtm_eigen(www, a, is_, s.nbc, s.nt, s.dtx, s.dx, s.dt, s.gx, np.ones(s.ng), s.source(),
                                  s.vp_ratio * vs, vs, s.isfs, s.fd_order, 0, s.nt_wf)
    else:
        cl, cm, il = e2drtm_eigend(www, a, is_, s.nbc, s.nt, s.dtx, s.dx, s.dt, s.gx, np.ones(s.ng), s.source(),
                                   s.vp_ratio * vs, vs, s.isfs, s.fd_order, 0, s.nt_wf)
    out.update(cl=np.asarray(cl, np.float64), cm=np.asarray(cm, np.float64), il=np.asarray(il, np.float64))
    return out


def _assemble(s, vs, per, keep_shots):
    """SWD.m:188-201 from the per-shot results in shot order: FP64 shot sums, the Vs gradient,
    smoothing and the misfit."""
    g = {k: np.zeros((s.nz, s.nx)) for k in ("cl", "cm", "il")}
    for p in per:
        for k in g:
            g[k] = g[k] + p[k]
    dk = -4 * vs * (g["cl"] / g["il"]) + 2 * vs * (g["cm"] / g["il"])  # SWD.m:199-200
    res_r = np.array([p["res_r"] for p in per])
    out = {"g_cl": g["cl"], "g_cm": g["cm"], "g_illum": g["il"], "dk_vs": smooth2a(dk, s.smooth_z, s.smooth_x),
           "res_r": res_r, "res_l": np.array([p["res_l"] for p in per]),
           "cr_pre_r": np.stack([p["crp_r"] for p in per], 1), "cr_pre_l": np.stack([p["crp_l"] for p in per], 1),
           "residual": float(np.nanmean(res_r)) if np.any(~np.isnan(res_r)) else float("nan")}
    if keep_shots:
        out["per_shot"] = per
    return out


def gradient_many(cases, field=0, FK=0):
    """SWD_single.m:171-201 for several surveys at once, on grids of any sizes: the forward of every
    shot of every survey runs as one batch (swd_staggerfd_single_batch: one launch per time step
    for all of them), the spectra, picks and adjoint sources per shot, then the adjoint of every
    shot as one batch (swd_e2drtm_single_batch), reading the forward's strain snapshots where the
    forward batch left them on the device.  cases: [(s, vs, cr0_r, cr0_l)].  Returns one dict per
    survey, equal to gradient(s, vs, cr0_r, cr0_l) of each (single path)."""
    from .fd import (e2drtm_mex_args, eigen_e2drtm_single_batch, eigen_staggerfd_single_batch, prep_model,
                     staggerfd_mex_args)
    fwd, keys, mats = [], [], []
    for c, (s, vs, _, _) in enumerate(cases):
        m = prep_model(s.nbc, s.dtx, s.dx, s.dt, s.vp_ratio * vs, vs, s.isfs, s.fd_order, True)
        mats.append(m)
        for is_ in range(1, s.ns + 1):
            args = staggerfd_mex_args(s.nbc, s.nt, s.dtx, s.dx, s.dt, int(s.sx[is_ - 1]), 1, s.gx, np.ones(s.ng),
                                      s.vp_ratio * vs, vs, s.isfs, s.fd_order, s.source_type, 0, s.nt_wf, True, m)
            fwd.append((*args, s.source()))
            keys.append((c, is_))
    seis, kept = eigen_staggerfd_single_batch(fwd, keep=True)
    per = [[] for _ in cases]
    adj = []
    on_device = dict.fromkeys(("fux", "fuz", "bwx", "bwz"))  # read from kept
    for (c, is_), (_, sw, _) in zip(keys, seis):
        s, vs, cr0_r, cr0_l = cases[c]
        out, a = _shot_adjoint_source(s, is_, sw, cr0_r, cr0_l, True, field, FK)
        per[c].append(out)
        adj.append(e2drtm_mex_args(on_device, a, s.nbc, s.nt, s.dtx, s.dx, s.dt, s.gx, np.ones(s.ng), s.vp_ratio * vs,
                                   vs, s.isfs, s.fd_order, 0, s.nt_wf, True, mats[c]))
    imgs = eigen_e2drtm_single_batch(adj, kept)
    del kept
    for (c, _), (cl, cm, il), out in zip(keys, imgs, [o for p in per for o in p]):
        out.update(cl=np.asarray(cl, np.float64), cm=np.asarray(cm, np.float64), il=np.asarray(il, np.float64))
    return [_assemble(cases[c][0], cases[c][1], per[c], False) for c in range(len(cases))]


def gradient(s, vs, cr0_r, cr0_l, single=True, keep_shots=False, field=0, FK=0):
    """SWD.m:171-201: shot sums in shot order (FP64), Vs gradient, smoothing, misfit."""
    per = [shot_gradient(s, is_, vs, cr0_r, cr0_l, single, field, FK) for is_ in range(1, s.ns + 1)]
    return _assemble(s, vs, per, keep_shots)
