"""TEST INFRASTRUCTURE ONLY -- the CPU oracle for the SWD gradient hot path.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this module; the product package ``swd_b200`` never does.

Parity status: the FD time loops are PINNED; the spectrum, pick and SoftMax steps are
UNPINNED.  The reference (zhangchang271/SWD) has no tests, golden vectors or stored
outputs, and MATLAB, Octave, Eigen and the MATLAB MEX headers are all absent.  Its two
C++ MEX sources are compiled unmodified into ``oracle/_ref`` against stand-ins for the
Eigen / MEX API subset they use (``oracle/swd_ref.py``), and tests/ check the C++
restatement of the FD loops against them bit for bit.  The ``.m`` steps (Radon, pick,
SoftMax gradient, assembly) have nothing that runs them here: every function below is a
restatement of a reference function, cited by file:line, in double precision like
MATLAB, so that the GPU path can be compared with it on identical seeded inputs.
Third-party semantics that the reference relies on but does not contain are restated
from their published definitions:

* MATLAB ``fft``/``ifft``: the plain DFT definition (numpy's pocketfft).
* MATLAB ``softmax`` (Deep Learning Toolbox): column-wise, max-shifted.
* MATLAB ``findpeaks`` (Signal Processing Toolbox), no options: a sample
  strictly larger than both neighbours; a flat peak is reported at its first
  index; signal endpoints are never peaks.
* MATLAB ``max``: first index of the maximum.
* MATLAB ``interp1`` 'linear' (NaN outside the sample range) and
  'nearest','extrap'.
* MATLAB ``round``: half away from zero.

The FD time loops live in ``oracle/swd_oracle.cpp`` (loaded through ctypes as
``oracle/_build/libswd_oracle.so``); ``fd_forward_np``/``fd_adjoint_np`` below
are a second, independent vectorised restatement of the same loops used to
cross-check the C++ one bit-for-bit on small grids.
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libswd_oracle.so")
_lib = None


def lib():
    """Load the compiled C++ oracle (``make -C oracle``)."""
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            raise RuntimeError(f"oracle library not built: {_LIB_PATH} (run make -C oracle)")
        L = ctypes.CDLL(_LIB_PATH)
        f32p = ctypes.POINTER(ctypes.c_float)
        f64p = ctypes.POINTER(ctypes.c_double)
        L.oracle_staggerfd_f32.argtypes = [f32p, ctypes.c_int] + [f32p] * 14
        L.oracle_staggerfd_f64.argtypes = [f64p, ctypes.c_int] + [f64p] * 14
        L.oracle_e2drtm_f32.argtypes = [f32p, ctypes.c_int] + [f32p] * 12 + [ctypes.c_int] + [f64p] * 3
        L.oracle_e2drtm_f64.argtypes = [f64p, ctypes.c_int] + [f64p] * 12 + [f64p] * 3
        for f in (L.oracle_staggerfd_f32, L.oracle_staggerfd_f64, L.oracle_e2drtm_f32, L.oracle_e2drtm_f64):
            f.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a):
    if a is None:
        return None
    t = ctypes.c_float if a.dtype == np.float32 else ctypes.c_double
    return a.ctypes.data_as(ctypes.POINTER(t))


def mround(x):
    """MATLAB round(): half away from zero."""
    x = float(x)
    r = math.floor(abs(x))
    if abs(x) - r >= 0.5:
        r += 1
    return int(math.copysign(r, x)) if r else 0


# --------------------------------------------------------------------------------------
# Model preparation (setup of the FD inputs)
# --------------------------------------------------------------------------------------

def calparam(vp, vs, den):
    """core/calparam.m:3-5."""
    ca = (vp ** 2) * den
    cm = (vs ** 2) * den
    cl = ca - 2 * cm
    return ca, cm, cl


def pad(p0, nbc, isfs, pad_top):
    """core/pad.m:3-8: edge replication, pad_top rows on top when isfs."""
    p = np.concatenate([np.repeat(p0[:, :1], nbc, 1), p0, np.repeat(p0[:, -1:], nbc, 1)], 1)
    top = pad_top if isfs else nbc
    return np.concatenate([np.repeat(p[:1, :], top, 0), p, np.repeat(p[-1:, :], nbc, 0)], 0)


def damp_circle(vmin, nzbc, nxbc, nbc, dx, isfs, pad_top):
    """core/damp_circle.m:5-71 (1-based loops restated 0-based)."""
    nz = nzbc - nbc - pad_top
    nx = nxbc - 2 * nbc
    a = (nbc - 1) * dx
    kappa = 3.0 * vmin * math.log(10000000.0) / (2.0 * a)
    r = (np.arange(nbc, dtype=np.float64) * dx) / a
    damp1d = kappa * (r * r)
    damp = np.zeros((nzbc, nxbc))
    for iz in range(pad_top, nz + pad_top):
        damp[iz, 0:nbc] = damp1d[::-1]
        damp[iz, nx + nbc:nx + 2 * nbc] = damp1d
    for ix in range(nbc, nx + nbc):
        damp[0:pad_top, ix] = 0.0 if isfs else damp1d[::-1]  # pad_top == nbc when isfs=0
        damp[nzbc - nbc:nzbc, ix] = damp1d
    def corner(iz1, ix1, cz, cx):
        d = math.sqrt((ix1 - cx) ** 2 + (iz1 - cz) ** 2)
        q = d / nbc
        return kappa * (q * q)
    if not isfs:
        for iz1 in range(1, pad_top + 1):
            for ix1 in range(1, nbc + 1):
                damp[iz1 - 1, ix1 - 1] = corner(iz1, ix1, pad_top + 1, nbc + 1)
            for ix1 in range(nx + nbc + 1, nxbc + 1):
                damp[iz1 - 1, ix1 - 1] = corner(iz1, ix1, pad_top + 1, nx + nbc)
    for iz1 in range(nz + pad_top + 1, nzbc + 1):
        for ix1 in range(1, nbc + 1):
            damp[iz1 - 1, ix1 - 1] = corner(iz1, ix1, nz + pad_top, nbc + 1)
        for ix1 in range(nx + nbc + 1, nxbc + 1):
            damp[iz1 - 1, ix1 - 1] = corner(iz1, ix1, nz + pad_top, nbc + nx)
    return damp


def ricker(f, dt, nt=None):
    """core/ricker.m:18-38."""
    nw = 2.2 / f / dt
    nw = 2 * math.floor(nw / 2) + 1
    nc = math.floor(nw / 2)
    k = np.arange(1, nw + 1, dtype=np.float64)
    alpha = (nc - k + 1) * f * dt * math.pi
    beta = alpha * alpha
    w0 = (1.0 - beta * 2) * np.exp(-beta)
    if nt is None:
        return w0
    if nt < len(w0):
        raise ValueError("nt is smaller than condition!")
    w = np.zeros(nt)
    w[: len(w0)] = w0
    return w


@dataclass
class FdInputs:
    """The padded material fields and input_vector a MEX call receives."""
    iv: np.ndarray
    temp: np.ndarray
    ca: np.ndarray
    cl: np.ndarray
    cm: np.ndarray
    cm1: np.ndarray
    b: np.ndarray
    b1: np.ndarray
    nzbc: int
    nxbc: int
    pad_top: int


def _prep(nbc, dtx, dx, dt, vp, vs, isfs, fd_order, dtype):
    """Shared model prep of staggerfd_eigen.m:37-107 and e2drtm_eigen.m:44-101."""
    nz, nx = vs.shape
    one = dtype.type(1)
    vp = np.asarray(vp, np.float64)
    vs = np.asarray(vs, np.float64)
    # calparam with den = ones(single|double): double squares, rounded to the class of den
    ca = (vp * vp).astype(dtype) * one
    cm = (vs * vs).astype(dtype) * one
    cl = (ca - dtype.type(2) * cm).astype(dtype)
    pad_top = (fd_order - 20) // 2 + 1 if isfs else nbc
    cm = pad(cm, nbc, isfs, pad_top)
    cl = pad(cl, nbc, isfs, pad_top)
    den = pad(np.ones((nz, nx), dtype), nbc, isfs, pad_top)
    nzbc, nxbc = cm.shape
    vmin = float(min(vp.min(), vs.min()))
    damp = damp_circle(vmin, nzbc, nxbc, nbc, dx, isfs, pad_top)
    temp = (1 - damp * dt).astype(dtype)
    if not isfs:
        raise NotImplementedError("isfs=0 leaves b1/cm1 undefined in the reference wrappers")
    ca = pad(ca, nbc, isfs, pad_top)
    r = pad_top - 1
    ca[r, :] = dtype.type(2) * cm[r, :]
    cl[r, :] = 0
    b = (dtype.type(dtx) / den).astype(dtype)
    b[r, :] = dtype.type(2) * b[r, :]
    return ca, cl, cm, cm.copy(), b, b.copy(), temp, nzbc, nxbc, pad_top


_SRC = {"p": 1, "s": 2, "s1": 3, "z": 4, "w": 5}


def fd_inputs(nbc, nt, dtx, dx, dt, sx, sz, gx, gz, vp, vs, isfs=1, fd_order=22, source_type="w",
              in_wf=5, single=True, adjoint=False):
    """Build the MEX inputs exactly as staggerfd_eigen.m:37-138 (forward) or e2drtm_eigen.m:44-121."""
    dtype = np.dtype(np.float32 if single else np.float64)
    ca, cl, cm, cm1, b, b1, temp, nzbc, nxbc, pad_top = _prep(nbc, dtx, dx, dt, vp, vs, isfs, fd_order, dtype)
    nz, nx = vs.shape
    gx = np.atleast_1d(np.asarray(gx, np.float64))
    gz = np.atleast_1d(np.asarray(gz, np.float64))
    ng = gx.size
    gxp, gzp = gx + nbc, gz + pad_top
    dg = gxp[1] - gxp[0] if ng > 1 else 1
    if adjoint:
        iv = [nt, nzbc, nxbc, dtx, ng, nbc, gzp[0], gxp[0], dg, fd_order, in_wf, nz, nx, dt]
    else:
        iv = [nt, nzbc, nxbc, dtx, ng, sz + pad_top, sx + nbc, gzp[0], gxp[0], dg,
              _SRC[source_type], fd_order, in_wf, nz, nx, 3]
    iv = np.asarray(iv, dtype)
    F = lambda a: np.asfortranarray(a, dtype)
    return FdInputs(iv, F(temp), F(ca), F(cl), F(cm), F(cm1), F(b), F(b1), nzbc, nxbc, pad_top)


def mex_staggerfd(inp: FdInputs, s, want_wf=True):
    """Call the C++ oracle with MEX arguments; returns (seismo_u, seismo_w, {fux,fuz,bwx,bwz})."""
    dt_ = inp.temp.dtype
    iv = inp.iv
    nt, ng, nz, nx, ntwf = int(iv[0]), int(iv[4]), int(iv[13]), int(iv[14]), int(iv[12])
    s = np.ascontiguousarray(np.asarray(s).reshape(-1)[:nt], dt_)
    su = np.zeros((nt, ng), dt_, order="F")
    sw = np.zeros((nt, ng), dt_, order="F")
    nrec = nt // ntwf
    wf = {k: (np.zeros((nz, nx, nrec), dt_, order="F") if want_wf else None) for k in ("fux", "fuz", "bwx", "bwz")}
    fn = lib().oracle_staggerfd_f32 if dt_ == np.float32 else lib().oracle_staggerfd_f64
    rc = fn(_p(np.ascontiguousarray(iv)), iv.size, _p(inp.temp), _p(inp.ca), _p(inp.cl), _p(inp.cm), _p(inp.cm1),
            _p(inp.b), _p(inp.b1), _p(s), _p(su), _p(sw), _p(wf["fux"]), _p(wf["fuz"]), _p(wf["bwx"]), _p(wf["bwz"]))
    if rc:
        raise ValueError(f"oracle_staggerfd rc={rc}")
    return su, sw, wf


def mex_e2drtm(inp: FdInputs, res, wf, accum_fp64=True):
    """Call the C++ adjoint oracle; returns (cl_img, cm_img, illum_div) as float64 arrays (nz x nx)."""
    dt_ = inp.temp.dtype
    iv = inp.iv
    nz, nx = int(iv[11]), int(iv[12])
    res = np.asfortranarray(res, dt_)
    outs = [np.zeros((nz, nx), np.float64, order="F") for _ in range(3)]
    W = [np.asfortranarray(wf[k], dt_) for k in ("fux", "fuz", "bwx", "bwz")]
    args = [_p(np.ascontiguousarray(iv)), iv.size, _p(inp.temp), _p(inp.ca), _p(inp.cl), _p(inp.cm), _p(inp.cm1),
            _p(inp.b), _p(inp.b1), _p(res)] + [_p(w) for w in W]
    if dt_ == np.float32:
        rc = lib().oracle_e2drtm_f32(*args, int(accum_fp64), *[_p(o) for o in outs])
    else:
        rc = lib().oracle_e2drtm_f64(*args, *[_p(o) for o in outs])
    if rc:
        raise ValueError(f"oracle_e2drtm rc={rc}")
    return tuple(outs)


def staggerfd_eigen(is_, nbc, nt, dtx, dx, dt, sx, sz, gx, gz, s, vp, vs, isfs=1, fd_order=22,
                    source_type="w", parameter_type=0, in_wf=5, single=True):
    """core/staggerfd_eigen.m:2-142 (single=False: staggerfd_eigend.m)."""
    inp = fd_inputs(nbc, nt, dtx, dx, dt, sx, sz, gx, gz, vp, vs, isfs, fd_order, source_type, in_wf, single)
    return mex_staggerfd(inp, s)


def e2drtm_eigen(wavefield_gradient, seismo_w, is_, nbc, nt, dtx, dx, dt, gx, gz, s, vp, vs, isfs=1,
                 fd_order=22, parameter_type=0, in_wf=5, single=True, accum_fp64=True):
    """core/e2drtm_eigen.m:8-123 (single=False: e2drtm_eigend.m)."""
    inp = fd_inputs(nbc, nt, dtx, dx, dt, 0, 0, gx, gz, vp, vs, isfs, fd_order, "w", in_wf, single, adjoint=True)
    return mex_e2drtm(inp, seismo_w, wavefield_gradient, accum_fp64)


# --------------------------------------------------------------------------------------
# Independent vectorised FD restatement (small grids; cross-checks the C++ oracle)
# --------------------------------------------------------------------------------------

def fd_forward_np(inp: FdInputs, s):
    """Vectorised restatement of core/eigen_staggerfd_single.cpp:207-357 (fd_order 22)."""
    T = inp.temp.dtype.type
    iv = inp.iv
    nt, NZ, NX, dtx = int(iv[0]), int(iv[1]), int(iv[2]), T(iv[3])
    ng, sz, sx, gz, gx, dg = int(iv[4]), int(iv[5]) - 1, int(iv[6]) - 1, int(iv[7]) - 1, int(iv[8]) - 1, int(iv[9])
    st, ntwf, nz, nx = int(iv[10]), int(iv[12]), int(iv[13]), int(iv[14])
    nbc = (NX - nx) // 2
    z = np.zeros((NZ, NX), inp.temp.dtype)
    uu, ww, xx, zz, xz = z.copy(), z.copy(), z.copy(), z.copy(), z.copy()
    fux, fuz, bwx, bwz = z.copy(), z.copy(), z.copy(), z.copy()
    te, b, b1, ca, cl, cm1 = (np.asarray(a) for a in (inp.temp, inp.b, inp.b1, inp.ca, inp.cl, inp.cm1))
    su = np.zeros((nt, ng), z.dtype)
    sw = np.zeros((nt, ng), z.dtype)
    wf = {k: np.zeros((nz, nx, nt // ntwf), z.dtype) for k in ("fux", "fuz", "bwx", "bwz")}
    C = (slice(1, NZ - 1), slice(1, NX - 1))
    S = lambda dz, dx_: (slice(1 + dz, NZ - 1 + dz), slice(1 + dx_, NX - 1 + dx_))
    cols = gx + dg * np.arange(ng)
    for it in range(nt):
        uu[C] = te[C] * uu[C] + b[C] * (((xx[S(0, 1)] - xx[C]) + xz[C]) - xz[S(-1, 0)])
        ww[C] = te[C] * ww[C] + b1[C] * (((xz[C] - xz[S(0, -1)]) + zz[S(1, 0)]) - zz[C])
        sv = T(s[it])
        if st == 5:
            ww[sz, sx] = sv
        elif st == 1:
            xx[sz, sx] += sv; zz[sz, sx] += sv
        elif st == 2:
            uu[sz, sx] += sv; uu[sz - 1, sx] -= sv; ww[sz, sx] += sv; ww[sz, sx + 1] += sv
        elif st == 3:
            uu[sz, sx] += sv; ww[sz, sx] += sv
        elif st == 4:
            zz[sz, sx] += sv
        fux[C] = uu[C] - uu[S(0, -1)]
        fuz[C] = uu[S(1, 0)] - uu[C]
        bwx[C] = ww[S(0, 1)] - ww[C]
        bwz[C] = ww[C] - ww[S(-1, 0)]
        xx = te * xx + (ca * fux + cl * bwz) * dtx
        zz = te * zz + (ca * bwz + cl * fux) * dtx
        xz = te * xz + (cm1 * (fuz + bwx)) * dtx
        zz[1, :] = 0
        sw[it] = ww[gz, cols]
        su[it] = uu[gz, cols]
        if it % ntwf == 0:
            k = it // ntwf
            for name, a in (("fux", fux), ("fuz", fuz), ("bwx", bwx), ("bwz", bwz)):
                wf[name][:, :, k] = a[2:2 + nz, nbc:nbc + nx]
    return su, sw, wf


def fd_adjoint_np(inp: FdInputs, res, wf, accum_fp64=True):
    """Vectorised restatement of core/eigen_e2drtm_single.cpp:181-283 (fd_order 22)."""
    dtp = inp.temp.dtype
    T = dtp.type
    iv = inp.iv
    nt, NZ, NX, dtx = int(iv[0]), int(iv[1]), int(iv[2]), T(iv[3])
    ng, nbc, gz, gx, dg = int(iv[4]), int(iv[5]), int(iv[6]) - 1, int(iv[7]) - 1, int(iv[8])
    ntwf, nz, nx, dt = int(iv[10]), int(iv[11]), int(iv[12]), T(iv[13])
    z = np.zeros((NZ, NX), dtp)
    uu, ww, xx, zz, xz = z.copy(), z.copy(), z.copy(), z.copy(), z.copy()
    te, b, b1, ca, cl, cm1 = (np.asarray(a) for a in (inp.temp, inp.b, inp.b1, inp.ca, inp.cl, inp.cm1))
    acc = np.float64 if accum_fp64 else dtp
    gcl, gcm, gil = (np.zeros((nz, nx), acc) for _ in range(3))
    C = (slice(1, NZ - 1), slice(1, NX - 1))
    S = lambda dz, dx_: (slice(1 + dz, NZ - 1 + dz), slice(1 + dx_, NX - 1 + dx_))
    cols = gx + dg * np.arange(ng)
    res = np.asarray(res, dtp)
    for it in range(nt - 2, -1, -1):
        du = ((ca[C] * xx[C] - ca[S(0, -1)] * xx[S(0, -1)]) + (cl[C] * zz[C] - cl[S(0, -1)] * zz[S(0, -1)])) + \
             (cm1[C] * xz[C] - cm1[S(-1, 0)] * xz[S(-1, 0)])
        dw = ((cl[S(1, 0)] * xx[S(1, 0)] - cl[C] * xx[C]) + (ca[S(1, 0)] * zz[S(1, 0)] - ca[C] * zz[C])) + \
             (cm1[S(0, 1)] * xz[S(0, 1)] - cm1[C] * xz[C])
        uu[C] = te[C] * uu[C] - b[C] * du
        ww[C] = te[C] * ww[C] - b1[C] * dw
        ww[gz, cols] = ww[gz, cols] + dt * res[it, :]
        xx[C] = te[C] * xx[C] - dtx * (uu[S(0, 1)] - uu[C])
        zz[C] = te[C] * zz[C] - dtx * (ww[C] - ww[S(-1, 0)])
        xz[C] = (te[C] * xz[C] - dtx * (uu[S(1, 0)] - uu[C])) - dtx * (ww[C] - ww[S(0, -1)])
        zz[1, :] = 0
        if it % ntwf == 0:
            k = it // ntwf
            fx, fz, bx, bz = (np.asarray(wf[n][:, :, k], dtp) for n in ("fux", "fuz", "bwx", "bwz"))
            I = (slice(2, 2 + nz), slice(nbc, nbc + nx))
            F = fx + bz
            tcl = F * (xx[I] + zz[I])
            tcm = T(2) * ((xx[I] * fx + zz[I] * bz) + T(0.5) * (xz[I] * (fz + bx)))
            til = F * F
            gcl = gcl + tcl.astype(acc)
            gcm = gcm + tcm.astype(acc)
            gil = gil + til.astype(acc)
    return gcl.astype(np.float64), gcm.astype(np.float64), gil.astype(np.float64)


# --------------------------------------------------------------------------------------
# Linear Radon transform (dispersion spectrum) and its saved state
# --------------------------------------------------------------------------------------

def radon_window(is_, b, offset, m, M, side):
    """Trace window of RTr.m:5-12 (side='r') or RTl.m:5-12 (side='l'); 1-based columns in order."""
    if side == "r":
        c0 = M * is_ - M + 1 + m
        nend = min(m + offset - 1 + M * is_ - M + 1, b)
        cols = list(range(c0, nend + 1))
    else:
        nend = M * is_ - M + 1 - offset - m
        if nend < 1:
            nend = 0
        cols = list(range(nend + 1, M * is_ - M + 1 - m + 1))
        cols = cols[::-1]  # fliplr
    return cols


def velocities(vmin, vmax, dv=1.0):
    """The phase-velocity axis: vmin:vmax in the reference (RTr.m:21); vmin:dv:vmax in general."""
    n = int(math.floor((vmax - vmin) / dv + 1e-9)) + 1
    return vmin + dv * np.arange(n, dtype=np.float64)


def radon(seismo, is_, df, dt, vmin, vmax, fmin, fmax, b, ds, offset, m, M, side, dv=1.0, FK=0):
    """RTrAD.m:2-35 / RTlAD.m:2-36 (ml is also RTr/RTl's output).  FK=1: the field drivers'
    variant that f-k filters the gather before the transform
    (fieldexamples/QadimahFault/core/RTrAD.m:14-16, RTlAD.m:15-17).

    Returns ml (np x npair, column-max normalised), dataLen and saveForBackward
    {mm (np x nf complex), ll0, lf, nf, ccn, ml_raw (np x npair), uxtpos (1-based cols, ascending)}.
    """
    cols = radon_window(is_, b, offset, m, M, side)
    uxt = np.asarray(seismo, np.float64)[:, [c - 1 for c in cols]]
    if FK == 1:
        uxt = fk_filter(uxt, dt, ds)
    noff = uxt.shape[1]
    x = (m + np.arange(noff, dtype=np.float64)) * ds
    ccn = int(math.trunc(1.0 / df / dt))
    nt = uxt.shape[0]
    u = np.zeros((ccn, noff))
    u[: min(nt, ccn)] = uxt[: min(nt, ccn)]
    d = np.fft.fft(u, axis=0).T  # noff x ccn
    lf = mround(fmin / df) + 1
    nf = mround(fmax / df) + 1
    pp = 1.0 / velocities(vmin, vmax, dv)
    w0 = 2.0 * math.pi * df
    th0 = w0 * np.outer(pp, x)                      # imag part of ll0 (np x noff)
    ll0 = 1j * th0
    mm = np.zeros((pp.size, nf), np.complex128)
    for j in range(lf, nf + 1):
        l = np.exp(1j * (th0 * (j - 1)))
        mm[:, j - 1] = l @ d[:, j - 1]
    mlraw = np.abs(mm[:, lf - 1:nf])
    ml = mlraw / mlraw.max(axis=0, keepdims=True)
    pos = sorted(cols)
    return ml, noff, dict(mm=mm, ll0=ll0, lf=lf, nf=nf, ccn=ccn, ml_raw=mlraw, uxtpos=pos, x=x)


# --------------------------------------------------------------------------------------
# Dispersion picking
# --------------------------------------------------------------------------------------

def findpeaks_locs(y):
    """1-based locations of MATLAB findpeaks(y) (no options), finite input."""
    y = np.asarray(y, np.float64)
    n = y.size
    locs = []
    k = 1
    while k < n - 1:
        if y[k] > y[k - 1]:
            j = k + 1
            while j < n and y[j] == y[k]:
                j += 1
            if j < n and y[j] < y[k]:
                locs.append(k + 1)
            k = j
        else:
            k += 1
    return locs


def _argmax1(v):
    return int(np.argmax(v)) + 1  # first index of the max, 1-based


def pickFDC1(ml, lp, fg, lfg, lpvalue=None):
    """core/pickFDC1.m:1-131; returns (cr_0 after interpolation, dvmin, dvmax, raw idx, chazhi).
    lpvalue: the seed pick of column lp given by the caller instead of the argmax of that column,
    which is all that fieldexamples/outcrop/core/pickFDCValue.m:1-131 changes (its :20)."""
    ml = np.asarray(ml, np.float64)
    if np.isnan(ml).any():
        raise ValueError("pickFDC1: NaN in the spectrum is not supported")
    a, b = ml.shape
    idx = np.zeros(b + 1, np.int64)          # 1-based arrays, index 0 unused
    dvmax = np.zeros(b + 1, np.int64)
    dvmin = np.zeros(b + 1, np.int64)
    qujian = np.full(b + 1, np.nan)
    chazhi = np.ones(b + 1, np.int64)
    col = lambda i: ml[:, i - 1]
    idx[lp] = _argmax1(col(lp)) if lpvalue is None else int(lpvalue)  # :19
    for i in range(lp - 1, 0, -1):                               # :21-77
        if idx[i + 1] == a:
            idx[i] = a
            dvmax[i] = dvmax[i + 1]
            dvmin[i] = dvmin[i + 1]
            continue
        if idx[i + 1] > a - 3:
            dvmax[i] = a
        else:
            mlmax = findpeaks_locs(-col(i)[idx[i + 1] - 1:a])
            dvmax[i] = a if not mlmax else idx[i + 1] + min(mlmax)
        if idx[i + 1] < 3:
            dvmin[i] = 1
        else:
            mlmin = findpeaks_locs(-col(i)[0:idx[i + 1]])
            dvmin[i] = 1 if not mlmin else max(mlmin)
        qujian[i] = dvmax[i] - dvmin[i]
        if qujian[i] > qujian[i + 1] * lfg:
            idx[i] = idx[i + 1]
            chazhi[i] = 0
            dvmax[i] = dvmax[i + 1]
            dvmin[i] = dvmin[i + 1]
            qujian[i] = dvmax[i] - dvmin[i]
        else:
            idx[i] = dvmin[i] + _argmax1(col(i)[dvmin[i] - 1:dvmax[i]]) - 1
    for i in range(lp + 1, b + 1):                               # :79-128
        if idx[i - 1] > a - 3:
            dvmax[i] = a
        else:
            mlmax = findpeaks_locs(-col(i)[idx[i - 1] - 1:a])
            dvmax[i] = a if not mlmax else idx[i - 1] + min(mlmax)
        if idx[i - 1] < 3:
            dvmin[i] = 1
        else:
            mlmin = findpeaks_locs(-col(i)[0:idx[i - 1]])
            dvmin[i] = 1 if not mlmin else max(mlmin)
        qujian[i] = dvmax[i] - dvmin[i]
        if qujian[i] > fg * qujian[i - 1]:
            idx[i] = idx[i - 1]
            chazhi[i] = 0
            dvmax[i] = dvmax[i - 1]
            dvmin[i] = dvmin[i - 1]
            qujian[i] = dvmax[i] - dvmin[i]
        else:
            idx[i] = dvmin[i] + _argmax1(col(i)[dvmin[i] - 1:dvmax[i]]) - 1
    cr = interp_picks(idx[1:], chazhi[1:])                       # :129-131
    return cr, dvmin[1:], dvmax[1:], idx[1:], chazhi[1:]


def interp_picks(idx, chazhi):
    """interp1(que, idx(que), 1:b, 'linear') then interp1(..., 'nearest', 'extrap') (pickFDC1.m:129-131)."""
    b = idx.size
    que = np.nonzero(chazhi == 1)[0] + 1
    if que.size < 2:
        raise ValueError("pickFDC1: interp1 needs at least two retained picks")
    q = np.arange(1, b + 1, dtype=np.float64)
    yv = idx[que - 1].astype(np.float64)
    out = np.full(b, np.nan)
    for t in range(b):
        xq = q[t]
        if xq < que[0] or xq > que[-1]:
            continue
        k = int(np.searchsorted(que, xq, side="right")) - 1
        if k >= que.size - 1:
            out[t] = yv[-1]
            continue
        x0, x1, y0, y1 = float(que[k]), float(que[k + 1]), yv[k], yv[k + 1]
        if xq == x0:
            out[t] = y0
        else:
            out[t] = y0 + (xq - x0) * ((y1 - y0) / (x1 - x0))
    lo, hi = int(que[0]) - 1, int(que[-1]) - 1
    out[:lo] = out[lo]
    out[hi + 1:] = out[hi]
    return out


def LHDispPick(ml, vmin, cr_0, method=1, ini=10):
    """core/LHDispPick.m:2-13."""
    if method == 1:
        cr, *_ = pickFDC1(ml, ini, 2, 4)
        cr_pre = cr + vmin
    else:
        cr_pre = np.argmax(ml, axis=0) + 1 + vmin
    res = float(np.mean((cr_pre - np.asarray(cr_0, np.float64)) ** 2))
    return res, cr_pre


def pickFDCValue(ml, lp, lpvalue, fg, lfg):
    """fieldexamples/outcrop/core/pickFDCValue.m:1-131: pickFDC1 seeded with idx(lp) = lpvalue."""
    return pickFDC1(ml, lp, fg, lfg, lpvalue=lpvalue)


def LHDispPick_field(ml, ml_raw, vmin, cr_0, method=1, variant=1):
    """The field-data LHDispPick variants, seeded at the global maximum of the unnormalised
    spectrum ml_raw (saveForBackward.mlr / .mll, RTrAD.m:34): [~,ini] = max(max(mlr)) is the first
    column holding the largest value, [~,iniP] = max(mlr(:,ini)) its first row of that value.

    variant 1: fieldexamples/outcrop/core/LHDispPick.m:2-25, pickFDCValue(ml, ini, iniP, 2, 4)
               for method 1, misfit over rows 15..end-15 (:24);
    variant 2: fieldexamples/QadimahFault/core/LHDispPick.m:2-41 with its mode 1, pickFDC1(ml,
               ini, 2, 4) whatever the method, misfit over rows 50..end-30 (:25).  That file also
               calls pickdisp_xl / CEDC when the window holds more than 100 traces; mode 1 does not
               use their results (and CEDC is not in the reference tree)."""
    raw = np.asarray(ml_raw, np.float64)
    ini = _argmax1(raw.max(axis=0))
    b = np.asarray(ml).shape[1]
    if variant == 1:
        if method == 1:
            cr, *_ = pickFDCValue(ml, ini, _argmax1(raw[:, ini - 1]), 2, 4)
            cr_pre = cr + vmin
        else:
            cr_pre = np.argmax(ml, axis=0) + 1 + vmin
        lo, hi = 15, b - 15
    elif variant == 2:
        cr, *_ = pickFDC1(ml, ini, 2, 4)
        cr_pre = cr + vmin
        lo, hi = 50, b - 30
    else:
        raise ValueError("variant must be 1 (outcrop) or 2 (QadimahFault)")
    d = cr_pre - np.asarray(cr_0, np.float64)
    res = float(np.mean(d[lo - 1:hi] ** 2)) if hi >= lo else float("nan")  # mean([]) is NaN
    return res, cr_pre


def norm_trace(data_in):
    """core/norm_trace.m:1-22: each trace (column) divided by its largest magnitude; the guard for
    an all-zero trace is commented out there, so such a trace becomes 0/0 = NaN."""
    d = np.asarray(data_in, np.float64)
    with np.errstate(invalid="ignore", divide="ignore"):
        return d / np.nanmax(np.abs(d), axis=0, keepdims=True)  # MATLAB's max skips NaN


def fk_filter(d, dt, dx):
    """core/fk_filter.m:1-302 (the same file in fieldexamples/*/core): the live code is the
    fixed dip filter of its "case 6".  The ns x ntr data are zero-padded to 2ns x 2ntr (:49-51),
    transformed by fft2 and fftshift (:52-53); in the shifted spectrum the quadrants
    (i <= nf/2, j <= nk/2) and (i > nf/2, j > nk/2) are zeroed (:283-289); fftshift again (an
    inverse shift for even sizes), real(ifft2) and the leading ns x ntr block (:293-296).
    dt and dx only set axes that the live code never uses (:56-67, :237)."""
    d = np.asarray(d, np.float64)
    ns, ntr = d.shape
    D = np.zeros((2 * ns, 2 * ntr))
    D[:ns, :ntr] = d
    D = np.fft.fftshift(np.fft.fft2(D))
    nf, nk = D.shape
    D[: nf // 2, : nk // 2] = 0.0
    D[nf // 2:, nk // 2:] = 0.0
    return np.real(np.fft.ifft2(np.fft.fftshift(D)))[:ns, :ntr]


# --------------------------------------------------------------------------------------
# SoftMax misfit gradient -> time-domain adjoint source
# --------------------------------------------------------------------------------------

def softmax_cols(z):
    """Column-wise softmax, max-shifted (MATLAB Deep Learning Toolbox softmax on an N-by-Q matrix)."""
    zm = z - z.max(axis=0, keepdims=True)
    e = np.exp(zm)
    return e / e.sum(axis=0, keepdims=True)


def normpdf_cols(npv, cr):
    """core/paddingMl_norm.m:1-9: column i is normpdf(1:np, cr(i), 16)."""
    x = np.arange(1, npv + 1, dtype=np.float64)[:, None]
    z = (x - np.asarray(cr, np.float64)[None, :]) / 16.0
    return np.exp(-0.5 * z * z) / (np.sqrt(2 * np.pi) * 16.0)


def adwd_side(nt, ng, npair, soft_arg_norm, grad_output, save, side, a_data_res, cr=None, limband=False):
    """One side of core/ADWDgrad_1.m:15-44 (right) / :47-77 (left), written into a_data_res.
    cr given: ADWDgrad_norm.m:22-23, the weights are normpdf around cr = cr_pre - vmin.
    limband: core/ADWDgradlimband.m:13-53, power-normalised weights and the 25-bin ramps."""
    lf, nf, ccn = save["lf"], save["nf"], save["ccn"]
    pos = save["uxtpos"]
    noff = len(pos)
    go = np.array(grad_output, np.float64).copy()
    go[go == 0] = 1
    if limband:  # ADWDgradlimband.m:20-31
        P = save["ml_raw"] ** soft_arg_norm
        P1 = soft_arg_norm * P ** (soft_arg_norm - 1)
        S = P.sum(axis=0, keepdims=True)
        N, N1 = P1 / S, P / S
        space = np.arange(1, N.shape[0] + 1, dtype=np.float64)[:, None]
        test3 = N * space - (space * N1).sum(axis=0, keepdims=True) * N
        gradml = test3 * 2 * go[None, :npair] * 1
    else:
        mlr = save["ml_raw"] ** (1.0 / 40.0)
        E = softmax_cols(mlr * soft_arg_norm) if cr is None else normpdf_cols(mlr.shape[0], cr)
        npv = E.shape[0]
        space = np.arange(1, npv + 1, dtype=np.float64)[:, None]
        mean_s = (space * E).sum(axis=0, keepdims=True)
        test3 = E * space - mean_s * E
        gradml = test3 * 2 * go[None, :npair] * soft_arg_norm
    mm = save["mm"][:, lf - 1:nf]
    with np.errstate(invalid="ignore", divide="ignore"):
        ph = mm / np.abs(mm)
    ph[np.isnan(ph)] = 0
    gm = ph * gradml
    th0 = save["ll0"].imag
    G = np.zeros((noff, ccn), np.complex128)
    for j in range(lf, nf + 1):
        K = np.exp(1j * (th0 * (j - 1)))
        G[:, j - 1] = K.conj().T @ gm[:, j - lf]
    if limband:  # ADWDgradlimband.m:41-48; ifft(.., ccn) drops columns past ccn
        if lf - 25 < 1:
            raise ValueError("ADWDgradlimband indexes column lf-25, which needs lf >= 26")
        for i in range(lf - 25, lf + 1):
            G[:, i - 1] = G[:, lf - 1] * ((i - lf + 25) / 25)
        for i in range(nf, nf + 26):
            if i <= ccn:
                G[:, i - 1] = G[:, nf - 1] * ((nf - i + 25) / 25)
    g = np.real(np.fft.ifft(G, ccn, axis=1))[:, :nt]      # noff x nt
    if side == "r":
        a_data_res[:, [p - 1 for p in pos]] = g.T
    else:
        # uxtposl ascending; row 1 of g is the source trace (fliplr); ADWDgrad_1.m:76
        a_data_res[:, [p - 1 for p in pos[:-1]]] = g[:0:-1, :].T
    return a_data_res


def ADWDgrad_norm(nt, ng, ns, npair, is_, w, m, M, SoftArgNorm, grad_outputr, grad_outputl, saver, savel, cr_r,
                  cr_l):
    """core/ADWDgrad_norm.m:1-102 (saveForBackward.cr_r / cr_l passed as cr_r / cr_l)."""
    a = np.zeros((nt, ng))
    if has_right(is_, ns, m, M, w):
        adwd_side(nt, ng, npair, SoftArgNorm, grad_outputr, saver, "r", a, cr_r)
    if has_left(is_, m, M, w):
        adwd_side(nt, ng, npair, SoftArgNorm, grad_outputl, savel, "l", a, cr_l)
    return a


def mlinspace(d1, d2, n):
    """MATLAB linspace(d1, d2, n): floor(n) points d1 + i*(d2-d1)/(n-1), the last one d2."""
    n = int(math.floor(n))
    if n < 1:
        return np.zeros(0)
    if n == 1:
        return np.array([float(d2)])
    y = d1 + np.arange(n, dtype=np.float64) * (d2 - d1) / (n - 1)
    y[-1] = d2
    return y


def weight_data_muti3(seismo_v_d, seismo_v, is_, dt, df, offset, dg, F1, w, M, m, ns, refsx, win, fmin, fmax,
                      cr_0, cr_0l, cr_pre_r, cr_pre_l, ind):
    """core/weight_data_muti3.m:1-122, the WD adjoint source (SWD.m:188, commented out there).

    Each side's traces are zero-padded to ntpad = floor(1/dt/df) samples and Fourier
    transformed; bins 2..win+1 are multiplied by -1i*dk*y/(2 pi) (F1=0, the predicted data
    seismo_v) or -1i*dk*y*exp(-1i*dk*y)/(2 pi) (F1=1, the observed data seismo_v_d), with
    dk = 2 pi f (cr_0 - cr_pre)/(cr_0 cr_pre) at bins ind..ind+npair-1 and 0 at the other
    bins up to win, and y the trace's offset in metres; bins ntpad-win+1..ntpad are set to the
    conjugates; the other bins keep the data's spectrum.  The inverse transform's first nt
    samples are the adjoint source.  The left side runs for is > round(w/M)+floor(m/M)+1
    (strictly greater, unlike ADWDgrad_1) and is written after the right side."""
    nt, b = np.shape(seismo_v_d)[:2]
    fre = 2 * np.pi * mlinspace(fmin, fmax, (fmax - fmin) / df + 1)  # :4
    npair = fre.size
    ntpad = int(math.floor(1 / dt / df))                               # :10
    if ind != math.floor(ind) or win != math.floor(win):
        raise ValueError("ind and win must be integers (they index deta_cc2)")
    ind, win = int(ind), int(win)
    if nt > ntpad or 2 * win >= ntpad or ind < 1 or ind + npair - 1 > win:
        raise ValueError("weight_data_muti3 needs nt <= ntpad, 2*win < ntpad and ind+npair-1 <= win")
    src = np.asarray(seismo_v_d if F1 == 1 else seismo_v, np.float64)
    out = np.zeros((nt, b))
    rs = int(refsx[is_ - 1])

    def filtered(c_first, c_last, y, cr0, crp):
        if c_last < c_first:
            raise ValueError(f"shot {is_}: empty WD window")
        dk = np.zeros(win)
        dk[ind - 1:ind - 1 + npair] = fre * (np.asarray(cr0, np.float64) - crp) / (cr0 * np.asarray(crp))
        temp = np.zeros((ntpad, c_last - c_first + 1))
        temp[:nt] = src[:, c_first - 1:c_last]
        spec = np.fft.fft(temp, axis=0)
        th = (-1j * dk[:, None]) * y[None, :]
        fac = (th * np.exp(th)) / np.pi / 2 if F1 == 1 else th / np.pi / 2   # :37-41
        for om in range(1, win + 1):                                         # :48-56
            spec[om] = spec[om] * fac[om - 1]
            spec[ntpad - om] = np.conj(spec[om])
        return np.real(np.fft.ifft(spec, axis=0))[:nt]

    if is_ <= ns - math.floor(m / M) - mround(w / M):                       # :21-68
        nend = min(m + offset - 1 + rs, b)
        newoffset = nend - (rs + m) + 1
        c0 = mround(m + rs)
        y = (m + mlinspace(0, newoffset - 1, newoffset)) * dg
        out[:, c0 - 1:nend] = filtered(c0, nend, y, cr_0, cr_pre_r)
    if is_ > mround(w / M) + math.floor(m / M) + 1:                         # :74-121
        nend = max(rs - offset - m, 0)
        newoffset = rs - m - nend
        y = (m + mlinspace(newoffset - 1, 0, newoffset)) * dg
        out[:, nend:rs - m] = filtered(nend + 1, rs - m, y, cr_0l, cr_pre_l)
    return out


def wd_direct(x, k_lo, fac, ntpad):
    """The same filter as weight_data_muti3 on one zero-padded trace, without FFTs: x plus
    (2/ntpad) Re sum_k (fac_k - 1) X_k exp(2 pi i k t / ntpad) over bins k = 1..len(fac).
    A cross-check of the restatement's bin bookkeeping."""
    x = np.asarray(x, np.float64)
    t = np.arange(x.size)
    k = np.arange(k_lo, k_lo + len(fac))
    E = np.exp(-2j * np.pi * np.outer(k, t) / ntpad)
    X = E @ x
    d = (np.asarray(fac) - 1) * X
    return x + 2.0 / ntpad * np.real(d @ E.conj())


def ADWDgradlimband(nt, ng, ns, npair, is_, w, m, M, SoftArgNorm, grad_outputr, grad_outputl, saver, savel):
    """core/ADWDgradlimband.m:1-102."""
    a = np.zeros((nt, ng))
    if has_right(is_, ns, m, M, w):
        adwd_side(nt, ng, npair, SoftArgNorm, grad_outputr, saver, "r", a, limband=True)
    if has_left(is_, m, M, w):
        adwd_side(nt, ng, npair, SoftArgNorm, grad_outputl, savel, "l", a, limband=True)
    return a


def has_right(is_, ns, m, M, w):
    return is_ <= ns - math.floor(m / M) - mround(w / M)


def has_left(is_, m, M, w):
    return is_ >= mround(w / M) + math.floor(m / M) + 1


def ADWDgrad_1(nt, ng, ns, npair, is_, w, m, M, SoftArgNorm, grad_outputr, grad_outputl, saver, savel):
    """core/ADWDgrad_1.m:1-81."""
    a = np.zeros((nt, ng))
    if has_right(is_, ns, m, M, w):
        adwd_side(nt, ng, npair, SoftArgNorm, grad_outputr, saver, "r", a)
    if has_left(is_, m, M, w):
        adwd_side(nt, ng, npair, SoftArgNorm, grad_outputl, savel, "l", a)
    return a


# --------------------------------------------------------------------------------------
# Gradient assembly
# --------------------------------------------------------------------------------------

def ADWDgrad_1_maxnorm(*args):
    """fieldexamples/outcrop/core/ADWDgrad_1.m:1-81: ADWDgrad_1 with the adjoint source divided by
    its largest magnitude at the end (:79), same arguments."""
    a = ADWDgrad_1(*args)
    with np.errstate(invalid="ignore", divide="ignore"):
        return a / np.nanmax(np.abs(a))


def smooth2a(A, Nr, Nc):
    """core/smooth2a.m:38-76: (2Nr+1)x(2Nc+1) box mean with shrinking edges; NaNs are left out of
    the sums and counts and stay NaN in the output."""
    A = np.array(A, np.float64)
    r, c = A.shape
    eL = (np.abs(np.arange(r)[:, None] - np.arange(r)[None, :]) <= Nr).astype(np.float64)
    eR = (np.abs(np.arange(c)[:, None] - np.arange(c)[None, :]) <= Nc).astype(np.float64)
    nan = np.isnan(A)
    A[nan] = 0
    nrm = eL @ (~nan).astype(np.float64) @ eR
    nrm[nan] = np.nan
    return (eL @ A @ eR) / nrm


def assemble(vs, g_cl, g_cm, g_illum, smoothZ=1, smoothX=2):
    """SWD.m:199-201: illumination normalisation, Vs gradient, smoothing."""
    g_cl = g_cl / g_illum
    g_cm = g_cm / g_illum
    dk = -4 * vs * g_cl + 2 * vs * g_cm
    return smooth2a(dk, smoothZ, smoothX)


# --------------------------------------------------------------------------------------
# Whole shot loops of SWD.m / SWD_single.m
# --------------------------------------------------------------------------------------

def _survey_fd(s, is_, vs, single=True, adjoint=False, vp=None):
    vp = s.vp_ratio * vs if vp is None else vp
    return fd_inputs(s.nbc, s.nt, s.dtx, s.dx, s.dt, int(s.sx[is_ - 1]), 1, s.gx, np.ones(s.ng),
                     vp, vs, s.isfs, s.fd_order, s.source_type, s.nt_wf, single, adjoint)


def _gno(s, is_):
    """Shot number of the is_-th shot of s in its whole survey (a subset keeps them, shot_no)."""
    no = getattr(s, "shot_no", None)
    return int(no[is_ - 1]) if no is not None else is_


def _ns(s):
    """Shots of the whole survey (a subset keeps the count, ns_total)."""
    return int(getattr(s, "ns_total", None) or s.ns)


def _refsx(s, dgc):
    """refsx of SWD.m:96 (receiver index of each source) over the whole survey's shot numbers."""
    r = np.zeros(_ns(s))
    r[[_gno(s, i) - 1 for i in range(1, s.ns + 1)]] = np.floor(np.asarray(s.sx) / dgc) + 1
    return r


def _sides(s, is_):
    g = _gno(s, is_)
    return has_right(g, _ns(s), s.m, s.M, s.w), has_left(g, s.m, s.M, s.w)


def _spectra(s, seis, is_, FK=0):
    out = {}
    r_on, l_on = _sides(s, is_)
    for side, on in (("r", r_on), ("l", l_on)):
        if on:
            out[side] = radon(seis, _gno(s, is_), s.df, s.dt, s.vmin, s.vmax, s.fmin, s.fmax, s.ng, s.ds, s.offset,
                              s.m, s.M, side, s.dv, FK)
    return out


def observed_curves(s, vs, single=True, vp=None):
    """SWD.m:150-162 (SWD_single.m in single precision): picks of the data of model vs."""
    npair = s.npair
    cr = np.ones((npair, s.ns))
    cl = np.ones((npair, s.ns))
    for is_ in range(1, s.ns + 1):
        _, sw, _ = mex_staggerfd(_survey_fd(s, is_, vs, single, vp=vp), s.source(), want_wf=False)
        sp = _spectra(s, sw.astype(np.float64), is_)
        if "r" in sp:
            cr[:, is_ - 1] = LHDispPick(sp["r"][0], s.vmin, cr[:, is_ - 1], 1, s.ini)[1]
        if "l" in sp:
            cl[:, is_ - 1] = LHDispPick(sp["l"][0], s.vmin, cl[:, is_ - 1], 1, s.ini)[1]
    return cr, cl


def _fd_pair(fd, single, accum_fp64):
    """The FD calls of a shot loop: this module's restatement (fd="oracle"), or the reference's
    own MEX sources built into oracle/_ref (fd="reference"; single precision, FP32 image sums)."""
    if fd == "oracle":
        return mex_staggerfd, lambda inp, res, wf: mex_e2drtm(inp, res, wf, accum_fp64)
    if fd != "reference" or not single or accum_fp64:
        raise ValueError("fd='reference' runs the single MEX with its FP32 image sums only")
    from oracle import swd_ref
    return swd_ref.mex_staggerfd, lambda inp, res, wf: tuple(
        a.astype(np.float64) for a in swd_ref.mex_e2drtm(inp, res, wf))


def shot_gradient(s, is_, vs, cr0_r, cr0_l, accum_fp64=False, single=True, vp=None, weight="softmax",
                  fd="oracle", field=0, FK=0):
    """SWD_single.m:172-193 for one shot: forward (FP32), spectra, picks, ADWDgrad_1, adjoint.
    single=False: SWD.m's double path (FP64 FD, adjoint source kept in double).  accum_fp64=False
    (default) sums the single path's images in FP32, as the reference's single MEX does.
    fd="reference" runs the FD steps on the reference's own MEX sources (oracle/_ref).
    field=1 / 2: the field-data flow (fieldexamples/outcrop/outcrop.m:168-196): norm_trace of the
    predicted gather (in the data's precision), the field picker variant, the max-normalised
    ADWDgrad_1 (fieldexamples/outcrop/core/ADWDgrad_1.m:79).  FK=1: the gathers are f-k filtered
    before the Radon transform (fieldexamples/QadimahFault/QademahSWD3.m:119, core/RTrAD.m:14-16);
    the adjoint source is built from the filtered spectra, with no filter in the backward pass, as
    there."""
    fwd, adj = _fd_pair(fd, single, accum_fp64)
    inp = _survey_fd(s, is_, vs, single, vp=vp)
    _, sw, wf = fwd(inp, s.source())
    if field:
        sw_n = norm_trace(sw.astype(np.float64))
        sw = sw_n.astype(np.float32) if single else sw_n
    sp = _spectra(s, sw.astype(np.float64), is_, FK)
    npair = s.npair
    out = {"res_r": np.nan, "res_l": np.nan, "crp_r": np.ones(npair), "crp_l": np.ones(npair)}
    def pick(sd, cr0):
        if field:  # sd = (ml, noff, saved state) as radon() returns it
            return LHDispPick_field(sd[0], sd[2]["ml_raw"], s.vmin, cr0, 1, field)
        return LHDispPick(sd[0], s.vmin, cr0, 1, s.ini)

    if "r" in sp:
        out["res_r"], out["crp_r"] = pick(sp["r"], cr0_r[:, is_ - 1])
    if "l" in sp:
        out["res_l"], out["crp_l"] = pick(sp["l"], cr0_l[:, is_ - 1])
    gr = out["crp_r"] - cr0_r[:, is_ - 1]
    gl = out["crp_l"] - cr0_l[:, is_ - 1]
    if weight == "wd":  # SWD.m:188 (F1 = 0), ind/win of SWD.m:124-127, refsx of SWD.m:96
        dgc = int(s.gx[1] - s.gx[0])
        ind = s.fmin / s.df + 1
        a = weight_data_muti3(sw, sw.astype(np.float64), _gno(s, is_), s.dt, s.df, s.offset, s.ds, 0, s.w, s.M, s.m,
                              _ns(s),
                              _refsx(s, dgc), npair + 2 * ind, s.fmin, s.fmax,
                              cr0_r[:, is_ - 1], cr0_l[:, is_ - 1], out["crp_r"], out["crp_l"], ind)
    elif weight == "gauss":  # SWD.m:178,184 keep cr_pre - vmin in saveForBackward
        a = ADWDgrad_norm(s.nt, s.ng, _ns(s), npair, _gno(s, is_), s.w, s.m, s.M, s.soft_arg_norm, gr, gl,
                          sp.get("r", (0, 0, None))[2], sp.get("l", (0, 0, None))[2], out["crp_r"] - s.vmin,
                          out["crp_l"] - s.vmin)
    else:
        a = (ADWDgrad_1_maxnorm if field else ADWDgrad_1)(s.nt, s.ng, _ns(s), npair, _gno(s, is_), s.w, s.m, s.M,
                                                          s.soft_arg_norm, gr, gl,
                       sp.get("r", (0, 0, None))[2], sp.get("l", (0, 0, None))[2])
    out["adj_src"] = a.astype(np.float32) if single else a
    ainp = _survey_fd(s, is_, vs, single, adjoint=True, vp=vp)
    out["cl"], out["cm"], out["il"] = adj(ainp, out["adj_src"], wf)
    return out


def gradient(s, vs, cr0_r, cr0_l, threads=1, accum_fp64=False, single=True, vp=None, weight="softmax",
             fd="oracle", field=0, FK=0):
    """SWD_single.m:171-201 (SWD.m with single=False) with the shot sum in FP64 in shot order
    (per-shot images as shot_gradient)."""
    from concurrent.futures import ThreadPoolExecutor
    shots = list(range(1, s.ns + 1))
    if threads > 1:
        with ThreadPoolExecutor(threads) as ex:
            per = list(ex.map(lambda i: shot_gradient(s, i, vs, cr0_r, cr0_l, accum_fp64, single, vp, weight, fd,
                                                      field, FK), shots))
    else:
        per = [shot_gradient(s, i, vs, cr0_r, cr0_l, accum_fp64, single, vp, weight, fd, field, FK) for i in shots]
    g = {k: np.zeros((s.nz, s.nx)) for k in ("cl", "cm", "il")}
    for p in per:
        for k in g:
            g[k] = g[k] + p[k]
    res_r = np.array([p["res_r"] for p in per])
    out = {"g_cl": g["cl"], "g_cm": g["cm"], "g_illum": g["il"],
           "dk_vs": assemble(vs, g["cl"], g["cm"], g["il"], s.smooth_z, s.smooth_x),
           "res_r": res_r, "res_l": np.array([p["res_l"] for p in per]),
           "cr_pre_r": np.stack([p["crp_r"] for p in per], 1), "cr_pre_l": np.stack([p["crp_l"] for p in per], 1),
           "residual": float(np.nanmean(res_r)), "per_shot": per}
    return out


def contract(freq, vel, off, spec):
    """Slant stack of RTrAD.m:20-26 with general axes, for a batch of shots:
    mm[s,f,p] = sum_x exp(1i*2*pi*freq[f]*off[x]/vel[p]) * spec[s,f,x]   (FP64)."""
    freq, vel, off = (np.asarray(a, np.float64) for a in (freq, vel, off))
    th = 2 * np.pi * freq[:, None, None] * off[None, None, :] / vel[None, :, None]  # [f,p,x]
    return np.einsum("fpx,sfx->sfp", np.exp(1j * th), np.asarray(spec, np.complex128))


def misfit(s, vs, cr0_r, cr0_l, single=True, vp=None):
    """SWD.m:215-228: forward-only misfit of a trial model, the mean of res_r over the shots
    that have a right side (res_r is only assigned for them, and they come first)."""
    res = []
    for is_ in range(1, s.ns + 1):
        if not _sides(s, is_)[0]:
            continue
        _, sw, _ = mex_staggerfd(_survey_fd(s, is_, vs, single, vp=vp), s.source(), want_wf=False)
        ml = radon(sw.astype(np.float64), _gno(s, is_), s.df, s.dt, s.vmin, s.vmax, s.fmin, s.fmax, s.ng, s.ds, s.offset,
                   s.m, s.M, "r", s.dv)[0]
        res.append(LHDispPick(ml, s.vmin, cr0_r[:, is_ - 1], 1, s.ini)[0])
    return float(np.mean(res))
