"""TEST INFRASTRUCTURE ONLY -- ctypes binding of the reference's own FD MEX kernels.

``oracle/_ref/`` holds the reference's ``core/eigen_staggerfd_single.cpp`` and
``core/eigen_e2drtm_single.cpp``, compiled UNMODIFIED from the reference tree by
``make -C oracle ref`` against the Eigen / MATLAB MEX stand-ins in
``oracle/ref_shim/`` (see ``oracle/ref_entry.cpp``).  They pin the restated oracle
(``oracle/swd_oracle.cpp``) and, through it, the GPU kernels: tests compare all three
bit for bit.

Only ``tests/`` and ``bench.py``'s reference leg may import this module.  The
libraries are built where the reference tree is present and travel with the
repository as built files; :func:`available` says whether they are here.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")
_FWD = os.path.join(REF_DIR, "libswdref_staggerfd_single.so")
_ADJ = os.path.join(REF_DIR, "libswdref_e2drtm_single.so")
_libs = {}

_f32p = ctypes.POINTER(ctypes.c_float)


def available() -> bool:
    return os.path.exists(_FWD) and os.path.exists(_ADJ)


def _load(path, name, argtypes):
    if path not in _libs:
        if not os.path.exists(path):
            raise RuntimeError(f"reference library not built: {path} (run make -C oracle ref)")
        L = ctypes.CDLL(path)
        f = getattr(L, name)
        f.argtypes = argtypes
        f.restype = ctypes.c_int
        _libs[path] = f
    return _libs[path]


def _fp(a):
    return a.ctypes.data_as(_f32p) if a is not None else None


def _f(a):
    return np.asfortranarray(a, np.float32)


def eigen_staggerfd_single(iv, temp, ca, cl, cm, cm1, b, b1, s, want_wf=True):
    """The reference MEX ``eigen_staggerfd_single(iv,temp,ca,cl,cm,cm1,b,b1,s)``
    (core/eigen_staggerfd_single.cpp:68-383); returns (seismo_u, seismo_w, {fux,fuz,bwx,bwz})."""
    fn = _load(_FWD, "swdref_eigen_staggerfd_single",
               [_f32p, ctypes.c_int, ctypes.c_int, ctypes.c_int] + [_f32p] * 8 + [ctypes.c_int]
               + [_f32p, _f32p, ctypes.c_size_t] + [_f32p] * 4 + [ctypes.c_size_t, ctypes.c_char_p, ctypes.c_int])
    iv = np.ascontiguousarray(iv, np.float32).reshape(-1)
    nt, ng, ntwf, nz, nx = int(iv[0]), int(iv[4]), int(iv[12]), int(iv[13]), int(iv[14])
    nzbc, nxbc = temp.shape
    s = np.ascontiguousarray(np.asarray(s, np.float32).reshape(-1))
    su = np.zeros((nt, ng), np.float32, order="F")
    sw = np.zeros((nt, ng), np.float32, order="F")
    nrec = nt // ntwf
    wf = {k: (np.zeros((nz, nx, nrec), np.float32, order="F") if want_wf else None)
          for k in ("fux", "fuz", "bwx", "bwz")}
    flds = [_f(a) for a in (temp, ca, cl, cm, cm1, b, b1)]
    err = ctypes.create_string_buffer(256)
    rc = fn(_fp(iv), iv.size, nzbc, nxbc, *[_fp(a) for a in flds], _fp(s), s.size, _fp(su), _fp(sw), su.size,
            _fp(wf["fux"]), _fp(wf["fuz"]), _fp(wf["bwx"]), _fp(wf["bwz"]), nz * nx * nrec, err, 256)
    if rc:
        raise RuntimeError(f"reference eigen_staggerfd_single rc={rc}: {err.value.decode()}")
    return su, sw, wf


def eigen_e2drtm_single(iv, temp, ca, cl, cm, cm1, b, b1, seismo_w, fux, fuz, bwx, bwz):
    """The reference MEX ``eigen_e2drtm_single(iv,temp,ca,cl,cm,cm1,b,b1,seismo_w,fux,fuz,bwx,bwz)``
    (core/eigen_e2drtm_single.cpp:67-297); returns (cl_img, cm_img, illum_div) as nz x nx float32."""
    fn = _load(_ADJ, "swdref_eigen_e2drtm_single",
               [_f32p, ctypes.c_int, ctypes.c_int, ctypes.c_int] + [_f32p] * 8 + [ctypes.c_int, ctypes.c_int]
               + [_f32p] * 4 + [ctypes.c_int] * 3 + [_f32p] * 3 + [ctypes.c_size_t, ctypes.c_char_p, ctypes.c_int])
    iv = np.ascontiguousarray(iv, np.float32).reshape(-1)
    nt, ntwf, nz, nx = int(iv[0]), int(iv[10]), int(iv[11]), int(iv[12])
    nrec = nt // ntwf
    nzbc, nxbc = temp.shape
    res = _f(seismo_w)
    if res.shape[0] != nt:
        raise ValueError("seismo_w must have nt rows")
    W = [_f(np.asarray(w).reshape(nz, nx, -1, order="F")[:, :, :nrec]) for w in (fux, fuz, bwx, bwz)]
    outs = [np.zeros((nz, nx), np.float32, order="F") for _ in range(3)]
    flds = [_f(a) for a in (temp, ca, cl, cm, cm1, b, b1)]
    err = ctypes.create_string_buffer(256)
    rc = fn(_fp(iv), iv.size, nzbc, nxbc, *[_fp(a) for a in flds], _fp(res), res.shape[0], res.shape[1],
            *[_fp(w) for w in W], nz, nx, nrec, *[_fp(o) for o in outs], nz * nx, err, 256)
    if rc:
        raise RuntimeError(f"reference eigen_e2drtm_single rc={rc}: {err.value.decode()}")
    return tuple(outs)


def mex_staggerfd(inp, s, want_wf=True):
    """Same call as ``oracle.swd_oracle.mex_staggerfd`` on an ``FdInputs`` (float32 only)."""
    nt = int(inp.iv[0])
    s = np.asarray(s, np.float32).reshape(-1)[:nt]
    return eigen_staggerfd_single(inp.iv, inp.temp, inp.ca, inp.cl, inp.cm, inp.cm1, inp.b, inp.b1, s, want_wf)


def mex_e2drtm(inp, res, wf):
    """Same call as ``oracle.swd_oracle.mex_e2drtm`` with FP32 image sums; float32 images."""
    return eigen_e2drtm_single(inp.iv, inp.temp, inp.ca, inp.cl, inp.cm, inp.cm1, inp.b, inp.b1, res,
                               wf["fux"], wf["fuz"], wf["bwx"], wf["bwz"])
