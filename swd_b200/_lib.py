"""ctypes binding of libswd.so (the CUDA kernels and their C ABI).

The library is built in-tree (``python -m swd_b200.build``).  There is no CPU
fallback: if the library is missing or no CUDA device is visible, calls raise.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libswd.so")

_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)
_i32p = ctypes.POINTER(ctypes.c_int)
_c_int = ctypes.c_int
_c_dbl = ctypes.c_double
_vp = ctypes.c_void_p


class RadonParams(ctypes.Structure):
    """swd_radon_params of include/swd.h."""
    _fields_ = [("df", ctypes.c_double), ("dt", ctypes.c_double), ("fmin", ctypes.c_double),
                ("fmax", ctypes.c_double), ("vmin", ctypes.c_double), ("vmax", ctypes.c_double),
                ("dv", ctypes.c_double), ("ds", ctypes.c_double), ("nt", ctypes.c_int), ("ng", ctypes.c_int),
                ("offset", ctypes.c_int), ("m", ctypes.c_int), ("M", ctypes.c_int), ("precision", ctypes.c_int)]


_rpp = ctypes.POINTER(RadonParams)

# name -> argtypes (all return int status unless listed in _RESTYPE)
_SIGS = {
    "swd_last_error": [],
    "swd_version": [],
    "swd_kernel_launches": [],
    "swd_staggerfd_single": [_f32p, _c_int] + [_f32p] * 14,
    "swd_staggerfd_single_batch": [_c_int, ctypes.c_void_p],
    "swd_e2drtm_single_batch": [_c_int, ctypes.c_void_p],
    "swd_staggerfd_single_batch_keep": [_c_int, ctypes.c_void_p, ctypes.c_void_p],
    "swd_e2drtm_single_batch_kept": [_c_int, ctypes.c_void_p, ctypes.c_void_p],
    "swd_fd_batch_free": [ctypes.c_void_p],
    "swd_staggerfd_double": [_f64p, _c_int] + [_f64p] * 14,
    "swd_e2drtm_single": [_f32p, _c_int] + [_f32p] * 15,
    "swd_e2drtm_single_f64out": [_f32p, _c_int] + [_f32p] * 12 + [_f64p] * 3,
    "swd_e2drtm_double": [_f64p, _c_int] + [_f64p] * 15,
    "swd_prep_model_single": [_c_int] * 5 + [_c_dbl] * 3 + [_f64p] * 2 + [_f32p] * 7,
    "swd_prep_model_double": [_c_int] * 5 + [_c_dbl] * 3 + [_f64p] * 2 + [_f64p] * 7,
    "swd_radon_sizes": [_rpp] + [_i32p] * 5,
    "swd_radon": [_rpp, _c_int, _c_int] + [_f64p] * 4 + [_i32p] * 2,
    "swd_pick": [_f64p, _c_int, _c_int, _c_dbl, _f64p, _c_int, _c_int, _f64p, _f64p],
    "swd_pick_noalloc": [ctypes.c_void_p, _c_int, _c_int, _c_dbl, ctypes.c_void_p, _c_int, _c_int,
                         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    "swd_adwdgrad": [_rpp, _c_int, _c_int, _c_int, _c_dbl] + [_f64p] * 8,
    "swd_adwdgrad_norm": [_rpp, _c_int, _c_int, _c_int, _c_dbl] + [_f64p] * 10,
    "swd_adwdgrad_limband": [_rpp, _c_int, _c_int, _c_int, _c_dbl] + [_f64p] * 8,
    "swd_adwdgrad_maxnorm": [_rpp, _c_int, _c_int, _c_int, _c_dbl] + [_f64p] * 8,
    "swd_pick_field": [_f64p, _f64p, _c_int, _c_int, _c_dbl, _f64p, _c_int, _c_int, _f64p, _f64p],
    "swd_norm_trace": [_f64p, _c_int, _c_int, _f64p],
    "swd_fk_filter": [_f64p, _c_int, _c_int, ctypes.c_double, ctypes.c_double, _f64p],
    "swd_wd_residual": [_c_int, _c_int, _f64p, _f64p, _c_int, _c_dbl, _c_dbl, _c_int, _c_dbl, _c_int, _c_int,
                        _c_dbl, _c_int, _c_int, _f64p, _c_int, _c_dbl, _c_dbl] + [_f64p] * 4 + [_c_int, _f64p],
}
_RESTYPE = {"swd_last_error": ctypes.c_char_p, "swd_kernel_launches": ctypes.c_uint64, "swd_fd_batch_free": None}

SWD_OK = 0
_STATUS = {1: "SWD_ERR_INVALID", 2: "SWD_ERR_UNSUPPORTED", 3: "SWD_ERR_CUDA", 4: "SWD_ERR_OOM",
           5: "SWD_ERR_CANCELLED", 6: "SWD_ERR_NUMERIC"}


class SwdError(RuntimeError):
    """A libswd call returned a non-zero status."""

    def __init__(self, fn, status, msg):
        super().__init__(f"{fn}: {_STATUS.get(status, status)}: {msg}")
        self.status = status


_lib = None


def lib():
    """The loaded library (raises if it is not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libswd.so is not built ({LIB_PATH}); run python -m swd_b200.build")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = _RESTYPE.get(name, ctypes.c_int)
        _lib = L
    return _lib


def declared_symbols():
    """Every C entry point the Python package binds (here and in engine.py)."""
    from .engine import ENGINE_SYMBOLS
    from .contract import CONTRACT_SYMBOLS
    from .serve import SERVER_SYMBOLS
    return list(_SIGS) + ENGINE_SYMBOLS + SERVER_SYMBOLS + CONTRACT_SYMBOLS


def call(name, *args):
    """Call an int-returning entry point and raise SwdError on failure."""
    rc = getattr(lib(), name)(*args)
    if rc != SWD_OK:
        raise SwdError(name, rc, lib().swd_last_error().decode())
    return rc


def ptr(a):
    """ctypes pointer to a numpy array's data (None passes NULL)."""
    if a is None:
        return None
    if a.dtype == np.float32:
        return a.ctypes.data_as(_f32p)
    if a.dtype == np.float64:
        return a.ctypes.data_as(_f64p)
    if a.dtype == np.int32:
        return a.ctypes.data_as(_i32p)
    raise TypeError(f"unsupported dtype {a.dtype}")


def kernel_launches() -> int:
    return int(lib().swd_kernel_launches())
