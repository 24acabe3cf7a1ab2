"""CPU checks of the C ABI: the library loads and exports every symbol include/swd.h declares."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    txt = open(os.path.join(ROOT, "include", "swd.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(swd_[a-z0-9_]+)\s*\(", txt)))


def test_header_declares_entry_points():
    names = _declared()
    assert "swd_staggerfd_single" in names and "swd_e2drtm_single" in names
    assert len(names) >= 8


def test_library_exports_every_declared_symbol():
    from swd_b200 import _lib
    L = _lib.lib()
    missing = [n for n in _declared() if not hasattr(L, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    from swd_b200 import _lib
    assert set(_declared()) <= set(_lib.declared_symbols())


def test_calls_validate_before_touching_the_gpu():
    """Argument errors are reported without a device (no CUDA call happens before validation)."""
    import numpy as np
    from swd_b200 import _lib
    iv = np.zeros(16, np.float32)
    iv[:] = [100, 10, 20, 1e-4, 5, 3, 5, 3, 3, 1, 5, 24, 5, 4, 10, 3]
    z = np.zeros(200, np.float32)
    with pytest.raises(_lib.SwdError) as e:
        _lib.call("swd_staggerfd_single", _lib.ptr(iv), 16, *[_lib.ptr(z)] * 14)
    assert e.value.status == 2  # fd_order 24: unsupported
    iv[11] = 22
    iv[0] = 101  # not a multiple of nt_wf
    with pytest.raises(_lib.SwdError) as e:
        _lib.call("swd_staggerfd_single", _lib.ptr(iv), 16, *[_lib.ptr(z)] * 14)
    assert e.value.status == 1


def test_fk_filter_validates_before_touching_the_gpu():
    import numpy as np
    from swd_b200 import _lib
    d = np.zeros((4, 3))
    for ns, ntr in ((0, 3), (4, 0), (4, 70000)):
        with pytest.raises(_lib.SwdError) as e:
            _lib.call("swd_fk_filter", _lib.ptr(d), ns, ntr, 1e-3, 0.5, _lib.ptr(d))
        assert e.value.status == 1


def test_staggerfd_batch_validates_before_touching_the_gpu():
    import ctypes

    import numpy as np
    from swd_b200 import _lib
    from swd_b200.fd import _FdJob
    with pytest.raises(_lib.SwdError) as e:
        _lib.call("swd_staggerfd_single_batch", 0, None)
    assert e.value.status == 1
    iv = np.zeros(16, np.float32)
    iv[:] = [100, 10, 20, 1e-4, 5, 3, 5, 3, 3, 1, 5, 24, 5, 4, 10, 3]  # fd_order 24: unsupported
    z = np.zeros(200, np.float32)
    jobs = (_FdJob * 1)(_FdJob(iv.ctypes.data, 16, *[z.ctypes.data] * 10, None, None, None, None))
    with pytest.raises(_lib.SwdError, match="job 0") as e:
        _lib.call("swd_staggerfd_single_batch", 1, ctypes.cast(jobs, ctypes.c_void_p))
    assert e.value.status == 2


def test_engine_options_validate_before_touching_the_gpu():
    """Out-of-range engine options are reported as such, before any CUDA call."""
    import ctypes
    from swd_b200 import _lib, configs
    from swd_b200.engine import EngineOpts, GradientEngine, survey_struct
    s = configs.tiny(nt=400, ns=2)
    for fs in (-1, 7):
        with pytest.raises(_lib.SwdError, match="fd_schedule must lie in 0..6") as e:
            GradientEngine(s, fd_schedule=fs)
        assert e.value.status == 1
    sc = survey_struct(s)
    for field, value, msg in (("image_precision", 2, "image_precision must be 0"),
                              ("adjoint_weight", 3, "adjoint_weight must be 0")):
        opts = EngineOpts()
        setattr(opts, field, value)
        h = ctypes.c_void_p()
        with pytest.raises(_lib.SwdError, match=msg):
            _lib.call("swd_engine_create", ctypes.byref(sc), ctypes.byref(opts), ctypes.byref(h))


def test_product_never_imports_the_oracle():
    pkg = os.path.join(ROOT, "swd_b200")
    for dp, _, fs in os.walk(pkg):
        for f in fs:
            if f.endswith((".py", ".cu", ".cuh", ".h", ".cpp")):
                src = open(os.path.join(dp, f)).read()
                assert "oracle" not in re.sub(r"(#|//).*", "", src).lower() or f == "build.py", f


def test_engine_cancel_rejects_a_null_engine():
    """swd_engine_cancel validates its argument on the host, before any CUDA call."""
    from swd_b200 import _lib
    from swd_b200.engine import _bind
    _bind()
    with pytest.raises(_lib.SwdError, match="null engine") as e:
        _lib.call("swd_engine_cancel", None)
    assert e.value.status == 1
