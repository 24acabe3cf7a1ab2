"""Build a mex/ shim against the MEX API stand-in and call it with numpy data (test infrastructure)."""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
LIBDIR = os.path.join(ROOT, "swd_b200", "lib")
_CLS = {np.dtype(np.float64): 6, np.dtype(np.float32): 7}
_DT = {6: np.float64, 7: np.float32}


class MexError(RuntimeError):
    pass


class Shim:
    def __init__(self, name, outdir):
        src = os.path.join(ROOT, "mex", name + ".c")
        so = os.path.join(outdir, name.replace("/", "_") + ".so")
        cmd = ["gcc", "-O1", "-std=c11", "-D_GNU_SOURCE", "-shared", "-fPIC", "-I", HERE, "-I",
               os.path.join(ROOT, "mex"), "-I", os.path.join(ROOT, "include"), src, os.path.join(HERE, "mexsim.c"),
               "-L", LIBDIR, "-lswd", "-Wl,-rpath," + LIBDIR, "-lm", "-o", so]
        subprocess.run(cmd, check=True, capture_output=True)
        L = ctypes.CDLL(so)
        vp = ctypes.c_void_p
        L.sim_numeric.restype = vp
        L.sim_numeric.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t), vp, vp]
        L.sim_struct.restype = vp
        L.sim_set_field.argtypes = [vp, ctypes.c_char_p, vp]
        for f in ("sim_class", "sim_complex", "sim_ndim", "sim_nfields"):
            getattr(L, f).argtypes = [vp]
        L.sim_dim.restype = ctypes.c_size_t
        L.sim_dim.argtypes = [vp, ctypes.c_int]
        L.sim_re.restype = vp
        L.sim_re.argtypes = [vp]
        L.sim_im.restype = vp
        L.sim_im.argtypes = [vp]
        L.sim_field_name.restype = ctypes.c_char_p
        L.sim_field_name.argtypes = [vp, ctypes.c_int]
        L.sim_field_value.restype = vp
        L.sim_field_value.argtypes = [vp, ctypes.c_int]
        L.sim_destroy.argtypes = [vp]
        L.sim_cell.restype = vp
        L.sim_cell.argtypes = [ctypes.c_size_t]
        L.sim_set_cell.argtypes = [vp, ctypes.c_size_t, vp]
        L.sim_get_cell.restype = vp
        L.sim_get_cell.argtypes = [vp, ctypes.c_size_t]
        L.sim_numel.restype = ctypes.c_size_t
        L.sim_numel.argtypes = [vp]
        L.sim_error.restype = ctypes.c_char_p
        L.sim_call.argtypes = [ctypes.c_int, ctypes.POINTER(vp), ctypes.c_int, ctypes.POINTER(vp)]
        self.L = L

    def _to_mx(self, x):
        if isinstance(x, list):  # a 1 x n cell array
            c = self.L.sim_cell(len(x))
            for i, v in enumerate(x):
                self.L.sim_set_cell(c, i, self._to_mx(v))
            return c
        if isinstance(x, dict):
            s = self.L.sim_struct()
            for k, v in x.items():
                self.L.sim_set_field(s, k.encode(), self._to_mx(v))
            return s
        a = np.asarray(x)
        if a.dtype not in _CLS and not np.iscomplexobj(a):
            a = a.astype(np.float64)
        cplx = np.iscomplexobj(a)
        if cplx:
            a = a.astype(np.complex128)
        shape = a.shape if a.ndim >= 2 else ((1, 1) if a.ndim == 0 else (a.size, 1))
        dims = (ctypes.c_size_t * len(shape))(*shape)
        re = np.asfortranarray((a.real if cplx else a).reshape(shape))
        im = np.asfortranarray(a.imag.reshape(shape)) if cplx else None
        cls = 6 if cplx else _CLS[a.dtype]
        return self.L.sim_numeric(cls, len(shape), dims, re.ctypes.data, im.ctypes.data if cplx else None)

    def _from_mx(self, p):
        L = self.L
        if L.sim_class(p) == 1:
            return [self._from_mx(L.sim_get_cell(p, i)) for i in range(L.sim_numel(p))]
        if L.sim_class(p) == 2:
            return {L.sim_field_name(p, k).decode(): self._from_mx(L.sim_field_value(p, k))
                    for k in range(L.sim_nfields(p))}
        dt = _DT[L.sim_class(p)]
        shape = tuple(L.sim_dim(p, i) for i in range(L.sim_ndim(p)))
        n = int(np.prod(shape))

        def grab(ptr):
            return np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(np.ctypeslib.as_ctypes_type(dt))),
                                         (n,)).copy().reshape(shape, order="F")
        re = grab(L.sim_re(p)) if n else np.zeros(shape, dt)
        if L.sim_complex(p):
            return re + 1j * (grab(L.sim_im(p)) if n else 0)
        return re

    def __call__(self, nlhs, *args):
        vp = ctypes.c_void_p
        prhs = (vp * max(1, len(args)))(*[self._to_mx(a) for a in args])
        plhs = (vp * max(1, nlhs))()
        rc = self.L.sim_call(nlhs, plhs, len(args), prhs)
        for i in range(len(args)):
            self.L.sim_destroy(prhs[i])
        if rc:
            raise MexError(self.L.sim_error().decode())
        outs = [self._from_mx(plhs[i]) for i in range(max(1, nlhs)) if plhs[i]]
        for i in range(max(1, nlhs)):
            if plhs[i]:
                self.L.sim_destroy(plhs[i])
        return outs
