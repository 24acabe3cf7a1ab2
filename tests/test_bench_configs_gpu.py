"""Parity at the configurations the benchmark times (GPU against the oracle).

* The 100 x 600 survey (132 x 660 padded cells, 600 receivers, dt 5e-5): shots 1, 48 and 96 of
  the 96, nt 3000, in the configurations bench.py runs: stored snapshots with the autotuner's
  pick on that survey (two steps per launch, 4 warps, 4 slots, 26-row chunks), checkpoints
  every 50 steps (the survey's stated checkpoint interval), and the column-pair kernels, both
  ways.  The reference is SWD_single.m's shot loop (oracle) on the reference's own FD MEX
  sources (oracle/_ref, fd="reference").
* The 400 x 3000 survey's grid (442 x 3080 padded, 1200 receivers every second column, dt
  2.5e-5): shots 2 and 120, nt 500, checkpoint mode with 60-row chunks under the two-shots-per-
  warp kernels (the autotuner's pick there) and the column-pair kernels.  The survey's 40 Hz
  Ricker pulse is 2200 samples long, so these 500 steps use a 400 Hz pulse: the grid, model,
  receivers, chunking and kernels are the benchmark's.
* The Radon contraction at 200 frequencies x 400 velocities x 600 offsets (4 shots) in
  split-BF16 against the oracle's FP64 slant stack.

Picks are compared exactly.  Image sums and gradients at 1e-6 relative L2: the GPU's FP64
direct DFT and the oracle's FFT differ by ~1e-13 and may flip the FP32 rounding of a few
adjoint-source samples (SWD_single.m:193).  The engine configurations must agree with each
other bit for bit.
"""
import dataclasses

import numpy as np
import pytest

from swd_b200 import configs, shots
from swd_b200.engine import GradientEngine

pytestmark = pytest.mark.gpu

TOL = 1e-6
KEYS = ("g_cl", "g_cm", "g_illum")


def _rel(a, b):
    return np.linalg.norm(np.ravel(a - b)) / np.linalg.norm(np.ravel(b))


def _check(out, ref):
    assert np.array_equal(out["cr_pre_r"], ref["cr_pre_r"]) and np.array_equal(out["cr_pre_l"], ref["cr_pre_l"])
    for k in KEYS:
        assert np.abs(ref[k]).max() > 0, k
        assert _rel(out[k], ref[k]) < TOL, (k, _rel(out[k], ref[k]))
    # dk_vs divides by g_illum (SWD.m:199), which is 0 in cells no shot reached in these short
    # runs; there 0/0 or x/0 and the NaN-skipping smoothing depend on the sign and zero-ness of
    # FP32-rounding-level image values, so the comparison covers the cells finite in both, which
    # must be nearly all of the reference's finite cells
    fin = np.isfinite(ref["dk_vs"])
    ok = fin & np.isfinite(out["dk_vs"])
    assert ok.sum() >= 0.99 * fin.sum()
    if ok.any():  # a run short enough to leave x/0 in every smoothing window has no finite cell
        assert _rel(out["dk_vs"][ok], ref["dk_vs"][ok]) < TOL


def _same_bits(outs):
    for o in outs[1:]:
        for k in KEYS + ("cr_pre_r", "cr_pre_l"):
            assert np.array_equal(o[k], outs[0][k]), k
        assert np.array_equal(o["dk_vs"], outs[0]["dk_vs"], equal_nan=True)


@pytest.fixture(scope="module")
def batched_case(O, R):
    s = shots.subset(configs.batched_c2(nt=3000), [1, 48, 96])
    cr0_r, cr0_l = O.observed_curves(s, s.vs_true)
    ref = O.gradient(s, s.vs, cr0_r, cr0_l, threads=3, fd="reference")
    return s, cr0_r, cr0_l, ref


def test_batched_100x600_benchmark_configurations(batched_case):
    s, cr0_r, cr0_l, ref = batched_case
    outs = []
    for kw in ({"snapshot_mode": 1, "fd_schedule": 3, "warps": 4, "ring_fwd": 4, "ring_adj": 4, "chunk_rows": 26},
               {"snapshot_mode": 2, "ckpt_interval": 50, "fd_schedule": 3, "warps": 4, "ring_fwd": 4, "ring_adj": 4,
                "chunk_rows": 26},
               {"snapshot_mode": 1, "fd_schedule": 6},
               {"snapshot_mode": 2, "ckpt_interval": 50, "fd_schedule": 6}):
        with GradientEngine(s, **kw) as e:
            e.set_observed(cr0_r, cr0_l)
            out = e.gradient(s.vp, s.vs)
            assert e.info["mode"] == kw["snapshot_mode"]
        _check(out, ref)
        outs.append(out)
    _same_bits(outs)


def test_large_400x3000_grid_configurations(O, R):
    s = dataclasses.replace(shots.subset(configs.large_c5(nt=500), [2, 120]), f0=400.0)
    cr0_r, cr0_l = O.observed_curves(s, s.vs_true)
    ref = O.gradient(s, s.vs, cr0_r, cr0_l, threads=2, fd="reference")
    outs = []
    for kw in ({"fd_schedule": 5, "chunk_rows": 60}, {"fd_schedule": 6, "chunk_rows": 60}):
        with GradientEngine(s, snapshot_mode=2, ckpt_interval=100, **kw) as e:
            e.set_observed(cr0_r, cr0_l)
            out = e.gradient(s.vp, s.vs)
            assert e.info["chunk_rows"] == 60
        _check(out, ref)
        outs.append(out)
    _same_bits(outs)


def test_radon_contraction_200x400x600_split_bf16(O):
    import torch

    from swd_b200.contract import Contraction
    rng = np.random.default_rng(21)
    freq, vel, off = np.linspace(3.0, 80.0, 200), np.linspace(80.0, 1200.0, 400), np.arange(600) * 0.5
    spec = (rng.standard_normal((4, 200, 600)) + 1j * rng.standard_normal((4, 200, 600))).astype(np.complex64)
    spec = spec.astype(np.complex128)
    ref = O.contract(freq, vel, off, spec)
    with Contraction(freq, vel, off, spec.shape[0], "bf16x2") as c:
        d_mm = torch.zeros(c.shape_out, dtype=torch.complex128, device="cuda")
        c.run(torch.from_numpy(spec).cuda(), d_mm)
        torch.cuda.synchronize()
        assert not c.timed_out()
        got = d_mm.cpu().numpy()
    err = _rel(got, ref)
    print("split-BF16 rel L2", err)
    assert np.all(np.isfinite(got)) and err < 2e-4
