"""B200-native SWD gradient hot path (sm_100a CUDA kernels behind the reference's interfaces).

Modules:
    fd        FD forward modelling / adjoint imaging (MEX and .m-wrapper interfaces)
    _lib      ctypes binding of libswd.so
"""
from ._lib import SwdError, kernel_launches, lib  # noqa: F401
from .fd import (  # noqa: F401
    e2drtm_eigen,
    e2drtm_eigend,
    eigen_e2drtm_double,
    eigen_e2drtm_single,
    eigen_staggerfd_double,
    eigen_staggerfd_single,
    prep_model,
    staggerfd_eigen,
    staggerfd_eigend,
)

__version__ = "0.1.0"
