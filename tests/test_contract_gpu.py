"""Batched Radon contraction (swd_contract_*) against the oracle's FP64 slant stack.

Tolerances (relative L2 over all outputs): FP64 1e-12; FP32 1e-5 (FP32 operands and sums
over the offsets); split-BF16 hi+lo 2e-4 (the dropped lo*lo products and the hi/lo
rounding, ~2^-17 per operand); hi+mid+lo 1e-5 (down to FP32 rounding of the operands).
Sizes pad every tile dimension: 200 velocities (2 tiles of 128), 70 offsets (3 stages of
32), 100 shots (2 tiles of 96).
"""
import numpy as np
import pytest

from swd_b200.contract import Contraction

TOL = {"fp64": 1e-12, "fp32": 1e-5, "bf16x2": 2e-4, "bf16x3": 1e-5}


def _case(seed=3, nf=7, np_=200, nx=70, ns=100, uniform=True):
    rng = np.random.default_rng(seed)
    freq = np.linspace(3.0, 80.0, nf)
    vel = np.linspace(80.0, 1200.0, np_)
    off = np.arange(nx) * 0.5 if uniform else np.sort(rng.uniform(0.0, 35.0, nx))
    spec = (rng.standard_normal((ns, nf, nx)) + 1j * rng.standard_normal((ns, nf, nx))).astype(np.complex64)
    return freq, vel, off, spec.astype(np.complex128)


def test_contraction_rejects_bad_axes():
    with pytest.raises(Exception):
        Contraction([10.0], [0.0, 100.0], [0.0], 1)
    with pytest.raises(Exception):
        Contraction([10.0], [100.0], [0.0], 0)


def test_oracle_contraction_is_the_reference_slant_stack(O):
    """The general-axis oracle equals RTrAD's formula ll0 = 1i*2*pi*df*(pp*x), l = exp(ll0*(j-1))
    at f = df*(j-1), pp = 1/v."""
    df, js, v, x = 1.0, np.arange(5, 12), np.arange(100.0, 160.0), np.arange(12) * 0.5
    spec = np.random.default_rng(0).standard_normal((1, js.size, x.size)) + 0j
    ll0 = 1j * 2 * np.pi * df * np.outer(1.0 / v, x)
    want = np.stack([np.exp(ll0 * (j - 1)) @ spec[0, k] for k, j in enumerate(js)])[None]
    np.testing.assert_allclose(O.contract(df * (js - 1), v, x, spec), want, rtol=1e-12, atol=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64", "fp32", "bf16x2", "bf16x3"])
def test_contraction_matches_oracle(O, prec):
    import torch
    freq, vel, off, spec = _case()
    ref = O.contract(freq, vel, off, spec)
    with Contraction(freq, vel, off, spec.shape[0], prec) as c:
        d_spec = torch.from_numpy(spec).cuda()
        d_mm = torch.full(c.shape_out, np.nan, dtype=torch.complex128, device="cuda")
        c.run(d_spec, d_mm)
        torch.cuda.synchronize()
        assert not c.timed_out()
        got = d_mm.cpu().numpy()
        c.run(d_spec, d_mm)  # a second run on the same tables gives the same bits
        torch.cuda.synchronize()
        got2 = d_mm.cpu().numpy()
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    print(prec, "rel L2", err)
    assert np.all(np.isfinite(got)) and err < TOL[prec]
    assert np.array_equal(got, got2)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["bf16x2", "bf16x3"])
def test_contraction_with_uneven_offsets_matches_oracle(O, prec):
    """General axes: offsets that are not evenly spaced (the engine's are)."""
    import torch
    freq, vel, off, spec = _case(seed=4, uniform=False)
    ref = O.contract(freq, vel, off, spec)
    with Contraction(freq, vel, off, spec.shape[0], prec) as c:
        d_mm = torch.full(c.shape_out, np.nan, dtype=torch.complex128, device="cuda")
        c.run(torch.from_numpy(spec).cuda(), d_mm)
        torch.cuda.synchronize()
        assert not c.timed_out()
        got = d_mm.cpu().numpy()
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    print(prec, "uneven offsets rel L2", err)
    assert np.all(np.isfinite(got)) and err < TOL[prec]
