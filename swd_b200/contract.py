"""Batched Radon contraction with general axes (swd_contract_* of libswd.so).

    c = Contraction(freq, vel, offset, ns, precision="bf16x2")
    c.run(d_spec, d_mm)     # complex128 CUDA tensors [ns, nf, nx] -> [ns, nf, np]

mm[s,f,p] = sum_x exp(i*2*pi*freq[f]*offset[x]/vel[p]) * spec[s,f,x]: the slant stack of
RTrAD.m:20-26 for many shots.  fp64 / fp32 run on CUDA cores, bf16x2 / bf16x3 on the tcgen05
tensor cores with split-BF16 operands and FP32 accumulation.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import call

PRECISION = {"fp64": 0, "fp32": 1, "bf16x2": 2, "bf16x3": 3}
CONTRACT_SYMBOLS = ["swd_contract_create", "swd_contract_run", "swd_contract_status", "swd_contract_flops",
                    "swd_contract_destroy"]

_dp = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p


def _bind():
    L = _lib.lib()
    if getattr(L, "_contract_bound", False):
        return L
    sigs = {
        "swd_contract_create": [ctypes.c_int, _dp, ctypes.c_int, _dp, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int,
                                ctypes.c_int, ctypes.POINTER(_vp)],
        "swd_contract_run": [_vp, _vp, _vp, _vp],
        "swd_contract_status": [_vp, ctypes.POINTER(ctypes.c_int)],
        "swd_contract_flops": [_vp, _dp, _dp],
        "swd_contract_destroy": [_vp],
    }
    for n, a in sigs.items():
        f = getattr(L, n)
        f.argtypes = a
        f.restype = ctypes.c_int
    L._contract_bound = True
    return L


class Contraction:
    def __init__(self, freq, vel, offset, ns, precision="fp64", device=0):
        _bind()
        self.freq, self.vel, self.off = (np.ascontiguousarray(np.asarray(a, np.float64)) for a in (freq, vel, offset))
        self.ns, self.precision = int(ns), precision
        h = _vp()
        call("swd_contract_create", self.freq.size, self.freq.ctypes.data_as(_dp), self.vel.size,
             self.vel.ctypes.data_as(_dp), self.off.size, self.off.ctypes.data_as(_dp), self.ns,
             PRECISION[precision], int(device), ctypes.byref(h))
        self._h = h

    @property
    def shape_in(self):
        return (self.ns, self.freq.size, self.off.size)

    @property
    def shape_out(self):
        return (self.ns, self.freq.size, self.vel.size)

    def run(self, d_spec, d_mm, stream=None):
        """d_spec, d_mm: contiguous complex128 CUDA tensors of shape_in / shape_out."""
        if tuple(d_spec.shape) != self.shape_in or tuple(d_mm.shape) != self.shape_out:
            raise ValueError(f"spec must be {self.shape_in} and mm {self.shape_out}")
        call("swd_contract_run", self._h, _vp(d_spec.data_ptr()), _vp(d_mm.data_ptr()),
             _vp(stream.cuda_stream if stream is not None else 0))

    def timed_out(self):
        t = ctypes.c_int()
        call("swd_contract_status", self._h, ctypes.byref(t))
        return bool(t.value)

    def flops(self):
        u, i = ctypes.c_double(), ctypes.c_double()
        call("swd_contract_flops", self._h, ctypes.byref(u), ctypes.byref(i))
        return u.value, i.value

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().swd_contract_destroy(self._h)
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
