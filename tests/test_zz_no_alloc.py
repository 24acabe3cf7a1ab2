"""swd_pick_noalloc (device pointers, static scratch) against swd_pick (host pointers, cudaMalloc'd
scratch) and against the oracle's LHDispPick restatement.

The picker's results are integers plus vmin, so the entry points must agree exactly; the
misfit is compared with the rel 1e-12 the other picker tests use.  Two calls in a row on
different spectra check that the shared scratch carries nothing from one call into the next.
The device's free memory must not move across a call.
"""
import ctypes

import numpy as np
import pytest

from swd_b200 import _lib, spectrum as SP

MAX_NPAIR = 2047  # SWD_PICK_NOALLOC_MAX_NPAIR in include/swd.h


def _spectrum(rng, np_, npair):
    ml = rng.random((np_, npair))
    c = np.linspace(0.6, 0.3, npair) * np_
    p = np.arange(np_)[:, None]
    return ml + 3.0 * np.exp(-0.5 * ((p - c[None, :]) / 4.0) ** 2)


def _dev(a):
    import torch
    return torch.from_numpy(np.asarray(a, np.float64).ravel(order="F").copy()).cuda()


def _vp(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _noalloc(ml, vmin, cr0, method, ini, stream=None, with_res=True):
    import torch
    np_, npair = ml.shape
    d_ml, d_cr0 = _dev(ml), _dev(cr0)
    d_cr = torch.zeros(npair, dtype=torch.float64, device="cuda")
    d_res = torch.full((1,), np.nan, dtype=torch.float64, device="cuda") if with_res else None
    torch.cuda.synchronize()
    s = ctypes.c_void_p(stream.cuda_stream if stream is not None else 0)
    _lib.call("swd_pick_noalloc", _vp(d_ml), np_, npair, float(vmin), _vp(d_cr0), int(method), int(ini),
              _vp(d_res), _vp(d_cr), s)
    torch.cuda.synchronize()
    return (float(d_res.cpu()[0]) if with_res else None), d_cr.cpu().numpy()


@pytest.mark.gpu
def test_noalloc_pick_matches_swd_pick_on_two_calls_in_a_row():
    import torch
    rng = np.random.default_rng(2024)
    cases = [(351, 56, 10, 1), (120, 33, 5, 1)]
    side = torch.cuda.Stream()
    for k, (np_, npair, ini, method) in enumerate(cases):
        ml = _spectrum(rng, np_, npair)
        cr0 = rng.integers(1, np_, npair).astype(float) + 100
        ref_res, ref_cr = SP.LHDispPick(ml, 100, cr0, method, ini)
        res, cr = _noalloc(ml, 100, cr0, method, ini, stream=side if k else None)
        assert np.array_equal(cr, ref_cr), k
        assert res == pytest.approx(ref_res, rel=1e-12, abs=1e-12), k


@pytest.mark.gpu
def test_noalloc_pick_without_res_and_plain_argmax():
    rng = np.random.default_rng(5)
    ml = _spectrum(rng, 200, 40)
    cr0 = np.full(40, 250.0)
    _, ref_cr = SP.LHDispPick(ml, 100, cr0, 1, 7)
    _, cr = _noalloc(ml, 100, cr0, 1, 7, with_res=False)
    assert np.array_equal(cr, ref_cr)
    ref_res2, ref_cr2 = SP.LHDispPick(ml, 100, cr0, 2, 1)
    res2, cr2 = _noalloc(ml, 100, cr0, 2, 1)
    assert np.array_equal(cr2, ref_cr2) and res2 == pytest.approx(ref_res2, rel=1e-12, abs=1e-12)


@pytest.mark.gpu
def test_noalloc_pick_rejects_npair_beyond_its_scratch():
    import torch
    npair = MAX_NPAIR + 1
    d_ml = torch.zeros(4 * npair, dtype=torch.float64, device="cuda")
    d_v = torch.zeros(npair, dtype=torch.float64, device="cuda")
    with pytest.raises(_lib.SwdError) as e:
        _lib.call("swd_pick_noalloc", _vp(d_ml), 4, npair, 100.0, _vp(d_v), 1, 1, None, _vp(d_v), None)
    assert e.value.status == 1 and "2047" in str(e.value)


@pytest.mark.gpu
def test_noalloc_pick_matches_the_oracle_and_leaves_free_memory_unchanged():
    import torch

    from oracle import swd_oracle as O
    rng = np.random.default_rng(77)
    ml = _spectrum(rng, 351, 56)
    cr0 = rng.integers(1, 351, 56).astype(float) + 100
    ref_res, ref_cr = O.LHDispPick(ml, 100, cr0, 1, 10)
    np_, npair = ml.shape
    d_ml, d_cr0 = _dev(ml), _dev(cr0)
    d_cr = torch.zeros(npair, dtype=torch.float64, device="cuda")
    d_res = torch.zeros(1, dtype=torch.float64, device="cuda")
    args = (_vp(d_ml), np_, npair, 100.0, _vp(d_cr0), 1, 10, _vp(d_res), _vp(d_cr), None)
    _lib.call("swd_pick_noalloc", *args)  # the first call on a device may load the module
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        _lib.call("swd_pick_noalloc", *args)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert np.array_equal(d_cr.cpu().numpy(), ref_cr)
    assert float(d_res.cpu()[0]) == pytest.approx(ref_res, rel=1e-12, abs=1e-12)
