"""GPU parity of the batched gradient engine against the oracle's shot loop (SWD_single.m:171-201).

Picks are integer decisions and must match exactly.  The GPU's FP64 direct DFT and the
oracle's FFT differ by ~1e-13 relative; the adjoint source is then rounded to FP32
(single(seismo_v_d1), SWD_single.m:193), where such differences flip the rounding of a few
samples by one FP32 ulp (6e-8).  Images and the Vs gradient are therefore compared at
1e-6 relative L2 (FP32-rounding level).  Batching, checkpointing and CUDA graphs must not
change a single bit.
"""
import numpy as np
import pytest

from swd_b200 import configs
from swd_b200.engine import GradientEngine

pytestmark = pytest.mark.gpu

TOL = 1e-6


def _rel(a, b):
    return np.linalg.norm(np.ravel(a - b)) / np.linalg.norm(np.ravel(b))


@pytest.fixture(scope="module")
def tiny_case(O):
    s = configs.tiny(nt=400, ns=5)
    cr0_r, cr0_l = O.observed_curves(s, s.vs_true)
    ref = O.gradient(s, s.vs, cr0_r, cr0_l)
    return s, cr0_r, cr0_l, ref


def test_observed_curves_exact(O, tiny_case):
    s, cr0_r, cr0_l, _ = tiny_case
    with GradientEngine(s) as e:
        r, l = e.observed_curves(s.vp_true, s.vs_true)
    assert np.array_equal(r, cr0_r) and np.array_equal(l, cr0_l)


@pytest.mark.parametrize("mode,batch,graphs", [(1, 0, True), (1, 2, False), (2, 0, True), (2, 3, True)])
def test_gradient_matches_oracle(O, tiny_case, mode, batch, graphs):
    s, cr0_r, cr0_l, ref = tiny_case
    with GradientEngine(s, snapshot_mode=mode, max_batch=batch, use_graphs=graphs, ckpt_interval=35) as e:
        e.set_observed(cr0_r, cr0_l)
        out = e.gradient(s.vp, s.vs)
        out2 = e.gradient(s.vp, s.vs)  # graph replay
    assert np.array_equal(out["cr_pre_r"], ref["cr_pre_r"]) and np.array_equal(out["cr_pre_l"], ref["cr_pre_l"])
    np.testing.assert_allclose(out["res_r"], ref["res_r"], rtol=1e-12, equal_nan=True)
    for k in ("g_cl", "g_cm", "g_illum", "dk_vs"):
        assert _rel(out[k], ref[k]) < TOL, k
        assert np.array_equal(out[k], out2[k]), k
    assert out["residual"] == pytest.approx(ref["residual"], rel=1e-12)


def test_modes_are_bit_identical(tiny_case):
    s, cr0_r, cr0_l, _ = tiny_case
    outs = []
    for kw in ({"snapshot_mode": 1}, {"snapshot_mode": 2, "ckpt_interval": 20}, {"snapshot_mode": 1, "max_batch": 1},
               {"snapshot_mode": 2},  # memory-optimal checkpoint interval
               {"snapshot_mode": 1, "use_graphs": False, "chunk_rows": 3},
               # two barriers per row (shared-memory ring), shapes and ring depths
               {"snapshot_mode": 1, "fd_schedule": 4}, {"snapshot_mode": 2, "ckpt_interval": 20, "fd_schedule": 4},
               {"snapshot_mode": 1, "fd_schedule": 4, "warps": 1, "cells": 2, "chunk_rows": 3},
               {"snapshot_mode": 1, "fd_schedule": 4, "warps": 2, "cells": 1, "ring_fwd": 6, "ring_adj": 8},
               # one barrier per row (velocities a row ahead): same bits in every mode and chunking
               {"snapshot_mode": 1, "fd_schedule": 1}, {"snapshot_mode": 2, "ckpt_interval": 20, "fd_schedule": 1},
               {"snapshot_mode": 1, "fd_schedule": 1, "chunk_rows": 3},
               {"snapshot_mode": 1, "fd_schedule": 1, "chunk_rows": 5, "ring_fwd": 6, "ring_adj": 6},
               {"snapshot_mode": 1, "fd_schedule": 1, "warps": 2, "cells": 1, "chunk_rows": 1},
               {"snapshot_mode": 1, "fd_schedule": 1, "warps": 4, "cells": 1, "chunk_rows": 2},
               # warp streaming (no shared memory): same bits
               {"snapshot_mode": 1, "fd_schedule": 2}, {"snapshot_mode": 2, "ckpt_interval": 20, "fd_schedule": 2},
               {"snapshot_mode": 1, "fd_schedule": 2, "chunk_rows": 1},
               {"snapshot_mode": 1, "fd_schedule": 2, "warps": 2, "chunk_rows": 3},
               {"snapshot_mode": 2, "fd_schedule": 2, "warps": 8, "chunk_rows": 2, "use_graphs": False},
               {"snapshot_mode": 1, "fd_schedule": 2, "ring_fwd": 6, "ring_adj": 8, "chunk_rows": 9},
               {"snapshot_mode": 2, "fd_schedule": 2, "warps": 8, "ring_fwd": 8, "ring_adj": 6, "chunk_rows": 5},
               # two time steps per launch: pairs end at checkpoints (odd and even intervals)
               {"snapshot_mode": 1, "fd_schedule": 3}, {"snapshot_mode": 2, "ckpt_interval": 35, "fd_schedule": 3},
               {"snapshot_mode": 2, "ckpt_interval": 20, "fd_schedule": 3, "chunk_rows": 1},
               {"snapshot_mode": 1, "fd_schedule": 3, "warps": 8, "ring_fwd": 6, "chunk_rows": 4},
               {"snapshot_mode": 1, "fd_schedule": 3, "warps": 2, "ring_fwd": 8, "ring_adj": 6, "chunk_rows": 2,
                "use_graphs": False},
               # two steps per launch, two shots per warp (5 shots: the last warp carries one shot twice)
               {"snapshot_mode": 1, "fd_schedule": 5}, {"snapshot_mode": 2, "ckpt_interval": 35, "fd_schedule": 5},
               {"snapshot_mode": 2, "ckpt_interval": 20, "fd_schedule": 5, "chunk_rows": 1},
               {"snapshot_mode": 1, "fd_schedule": 5, "warps": 2, "ring_fwd": 6, "chunk_rows": 3, "max_batch": 2},
               {"snapshot_mode": 1, "fd_schedule": 5, "ring_adj": 6, "chunk_rows": 2, "max_batch": 3,
                "use_graphs": False},
               # two columns per lane in packed FP32 pairs, two steps per launch (one step for odd spans)
               {"snapshot_mode": 1, "fd_schedule": 6}, {"snapshot_mode": 2, "ckpt_interval": 35, "fd_schedule": 6},
               {"snapshot_mode": 2, "ckpt_interval": 20, "fd_schedule": 6, "chunk_rows": 1},
               {"snapshot_mode": 1, "fd_schedule": 6, "warps": 2, "ring_fwd": 6, "chunk_rows": 3, "max_batch": 2},
               {"snapshot_mode": 1, "fd_schedule": 6, "warps": 8, "ring_adj": 4, "chunk_rows": 2, "max_batch": 3,
                "use_graphs": False},
               {"snapshot_mode": 2, "ckpt_interval": 35, "fd_schedule": 6, "warps": 4, "ring_fwd": 6, "ring_adj": 6,
                "chunk_rows": 5}):
        with GradientEngine(s, **kw) as e:
            e.set_observed(cr0_r, cr0_l)
            outs.append(e.gradient(s.vp, s.vs))
    for o in outs[1:]:
        for k in ("g_cl", "g_cm", "g_illum", "dk_vs", "cr_pre_r"):
            assert np.array_equal(o[k], outs[0][k]), k


@pytest.mark.parametrize("sched", [0, 2, 5, 6])
def test_warp_chunks_are_capped_at_60_rows(sched):
    """The warp schedules mark a chunk's checked rows in a 64-bit mask, so their chunks are at
    most 60 rows: a 70-row grid asked for 500-row chunks runs 60 + 10 rows and gives the bits
    of the two-barrier schedule (which has no such cap)."""
    s = configs.tiny(nz=62, nx=24, nt=400, ns=3)
    outs = []
    for kw in ({"fd_schedule": 4}, {"fd_schedule": sched, "chunk_rows": 500}):
        with GradientEngine(s, snapshot_mode=1, **kw) as e:
            if kw["fd_schedule"] != 4:
                assert e.info["nzbc"] - 2 > 60 and e.info["chunk_rows"] == 60
            r, l = e.observed_curves(s.vp_true, s.vs_true)
            e.set_observed(r, l)
            outs.append(e.gradient(s.vp, s.vs))
    for k in ("g_cl", "g_cm", "g_illum", "dk_vs", "cr_pre_r"):
        assert np.array_equal(outs[1][k], outs[0][k]), k


@pytest.mark.parametrize("sched", [1, 2, 3, 4, 5, 6])
def test_other_schedules_on_the_plain_survey_match_the_oracle(O, sched):
    """The one-barrier (1), warp-streaming (2), two-steps-per-launch (3, the default),
    two-barrier (4) and two-shots-per-warp (5) schedules against the oracle on the 30 x 120
    survey (source near the top, receivers on the free-surface row, several chunks)."""
    s = configs.plain_c1(ns=3, nt=1000)
    cr0_r, cr0_l = O.observed_curves(s, s.vs_true)
    ref = O.gradient(s, s.vs, cr0_r, cr0_l)
    with GradientEngine(s, fd_schedule=sched, chunk_rows=7) as e:
        assert e.info["fd_schedule"] == sched
        e.set_observed(cr0_r, cr0_l)
        out = e.gradient(s.vp, s.vs)
    assert np.array_equal(out["cr_pre_r"], ref["cr_pre_r"])
    for k in ("g_cl", "g_cm", "g_illum", "dk_vs"):
        assert _rel(out[k], ref[k]) < TOL, k


def test_misfit_pass_matches_gradient_picks(tiny_case):
    s, cr0_r, cr0_l, ref = tiny_case
    with GradientEngine(s) as e:
        e.set_observed(cr0_r, cr0_l)
        m = e.misfit(s.vp, s.vs)
    assert np.array_equal(m["cr_pre_r"], ref["cr_pre_r"])
    np.testing.assert_allclose(m["res_r"], ref["res_r"], rtol=1e-12, equal_nan=True)


def test_plain_30x120_gradient(O):
    s = configs.plain_c1()
    cr0_r, cr0_l = O.observed_curves(s, s.vs_true)
    ref = O.gradient(s, s.vs, cr0_r, cr0_l, threads=8)
    with GradientEngine(s) as e:
        r, l = e.observed_curves(s.vp_true, s.vs_true)
        assert np.array_equal(r, cr0_r) and np.array_equal(l, cr0_l)
        e.set_observed(cr0_r, cr0_l)
        out = e.gradient(s.vp, s.vs)
    assert np.array_equal(out["cr_pre_r"], ref["cr_pre_r"])
    for k in ("g_cl", "g_cm", "g_illum", "dk_vs"):
        assert _rel(out[k], ref[k]) < TOL, (k, _rel(out[k], ref[k]))
    assert out["residual"] == pytest.approx(ref["residual"], rel=1e-12)


def test_sharded_engines_sum_to_the_full_survey(tiny_case):
    """Shots split over two engines (two ranks' shares, run one after the other on one GPU):
    picks and misfits per shot are identical and the FP64 shot sums add up to the full ones."""
    import torch

    from swd_b200 import shots
    s, cr0_r, cr0_l, _ = tiny_case
    with GradientEngine(s) as e:
        e.set_observed(cr0_r, cr0_l)
        full = e.gradient(s.vp, s.vs)
    n = s.nz * s.nx
    d_vp = torch.from_numpy(np.ascontiguousarray(s.vp.T)).cuda()
    d_vs = torch.from_numpy(np.ascontiguousarray(s.vs.T)).cuda()
    total = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    rsum, rcnt = 0.0, 0
    for rank in range(2):
        mine = shots.shard(s.ns, 2, rank)
        local = shots.subset(s, mine)
        with GradientEngine(local) as e:
            e.set_observed(cr0_r[:, mine - 1], cr0_l[:, mine - 1])
            part = e.gradient(s.vp, s.vs)
            assert np.array_equal(part["cr_pre_r"], full["cr_pre_r"][:, mine - 1])
            assert np.array_equal(part["cr_pre_l"], full["cr_pre_l"][:, mine - 1])
            np.testing.assert_array_equal(part["res_r"], full["res_r"][mine - 1])
            g = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
            a, c = e.shot_sums_device(d_vp, d_vs, g)
            torch.cuda.synchronize()
            total += g
            rsum, rcnt = rsum + a, rcnt + c
    t = total.cpu().numpy().reshape(3, s.nz, s.nx)
    for k, key in enumerate(("g_cl", "g_cm", "g_illum")):
        np.testing.assert_allclose(t[k], full[key], rtol=1e-12, atol=1e-300 + 1e-14 * np.abs(full[key]).max())
    assert rsum / rcnt == pytest.approx(full["residual"], rel=1e-12)


@pytest.mark.parametrize("mode", [1, 2])
def test_autotuned_engine_is_bit_identical(tiny_case, mode):
    """The autotuner only picks among variants that give the same bits; it reports what it timed."""
    s, cr0_r, cr0_l, _ = tiny_case
    outs = []
    for tune in (False, True):
        with GradientEngine(s, snapshot_mode=mode, ckpt_interval=35, autotune=tune) as e:
            e.set_observed(cr0_r, cr0_l)
            outs.append(e.gradient(s.vp, s.vs))
            if tune:
                assert e.info["tuned_fwd_us"] > 0 and e.info["tuned_adj_us"] > 0
                assert (e.info["warps"], e.info["cells"]) in [(3, 1), (2, 1), (4, 1), (1, 2), (8, 1)]
    for k in ("g_cl", "g_cm", "g_illum", "dk_vs", "cr_pre_r", "cr_pre_l"):
        assert np.array_equal(outs[0][k], outs[1][k]), k


@pytest.mark.parametrize("survey", ["tiny", "plain"])
def test_split_bf16_radon_in_the_engine(tiny_case, survey, O):
    """radon_precision='bf16x2': the forward contraction on the tensor cores, with the picker
    certifying every gather (a decision within 1e-4 of the column maximum sends the gather to the
    FP64 contraction and is picked again).  Picks are identical to the FP64 engine's -- also on
    the 30 x 120 survey, where uncertified split-BF16 spectra moved one pick in 672 -- and the
    gradient stays within the 1e-4 gradient tolerance."""
    if survey == "tiny":
        s, cr0_r, cr0_l, _ = tiny_case
    else:
        s = configs.plain_c1()
        cr0_r, cr0_l = O.observed_curves(s, s.vs_true)
    outs, stats = [], None
    for prec in ("fp64", "bf16x2"):
        with GradientEngine(s, radon_precision=prec) as e:
            e.set_observed(cr0_r, cr0_l)
            outs.append(e.gradient(s.vp, s.vs))
            if prec == "bf16x2":
                stats = e.radon_stats()
    a, b = outs
    print(survey, "recomputed in FP64", stats, "dk rel L2", _rel(b["dk_vs"], a["dk_vs"]))
    assert np.array_equal(a["cr_pre_r"], b["cr_pre_r"]) and np.array_equal(a["cr_pre_l"], b["cr_pre_l"])
    assert stats["gathers"] > 0 and stats["recomputed_fp64"] <= stats["gathers"]
    assert _rel(b["dk_vs"], a["dk_vs"]) < 1e-4


def test_gaussian_adjoint_weight_matches_oracle(tiny_case):
    """adjoint_weight='gauss' (ADWDgrad_norm) in the engine against the oracle's shot loop."""
    from oracle import swd_oracle as O
    s, cr0_r, cr0_l, _ = tiny_case
    ref = O.gradient(s, s.vs, cr0_r, cr0_l, weight="gauss")
    with GradientEngine(s, adjoint_weight="gauss") as e:
        e.set_observed(cr0_r, cr0_l)
        out = e.gradient(s.vp, s.vs)
    assert np.array_equal(out["cr_pre_r"], ref["cr_pre_r"])
    for k in ("g_cl", "g_cm", "g_illum", "dk_vs"):
        assert _rel(out[k], ref[k]) < TOL, k


def test_wd_adjoint_source_matches_oracle(tiny_case):
    """adjoint_weight='wd' (weight_data_muti3, SWD.m:188) in the engine against the oracle's shot loop."""
    from oracle import swd_oracle as O
    import dataclasses
    s, cr0_r, cr0_l, _ = tiny_case
    # fmin 50: ind = fmin/df+1 = 3 is an index (fmin 40 gives 2.6, which the reference cannot index
    # with); the Radon bins round(fmin/df)+1 .. are those of fmin 40, so the observed curves hold
    s = dataclasses.replace(s, fmin=50.0)
    ref = O.gradient(s, s.vs, cr0_r, cr0_l, weight="wd")
    with GradientEngine(s, adjoint_weight="wd") as e:
        e.set_observed(cr0_r, cr0_l)
        out = e.gradient(s.vp, s.vs)
    assert np.array_equal(out["cr_pre_r"], ref["cr_pre_r"])
    for k in ("g_cl", "g_cm", "g_illum", "dk_vs"):
        assert _rel(out[k], ref[k]) < TOL, k


@pytest.mark.parametrize("sched,mode,prec", [(0, 1, "fp32"), (0, 2, "fp32"), (4, 1, "fp32"), (5, 2, "fp32"),
                                            (6, 1, "fp32"), (6, 2, "fp32"), (0, 2, "fp64"), (4, 1, "fp64"),
                                            (5, 1, "fp64"), (6, 1, "fp64"), (6, 2, "fp64")])
def test_image_sums_match_the_oracle(O, tiny_case, sched, mode, prec):
    """image_precision='fp32' (the default) sums each shot's imaging terms in FP32, as the
    reference's single MEX does, and 'fp64' in FP64; against the oracle's shot loop with the same
    per-shot accumulation the shot sums come out identical."""
    s, cr0_r, cr0_l, _ = tiny_case
    ref = O.gradient(s, s.vs, cr0_r, cr0_l, accum_fp64=prec == "fp64")
    with GradientEngine(s, image_precision=prec, fd_schedule=sched, snapshot_mode=mode, ckpt_interval=35) as e:
        e.set_observed(cr0_r, cr0_l)
        out = e.gradient(s.vp, s.vs)
    assert np.array_equal(out["cr_pre_r"], ref["cr_pre_r"])
    for k in ("g_cl", "g_cm", "g_illum"):
        if prec == "fp32":
            assert np.array_equal(out[k], ref[k]), k
        else:
            assert _rel(out[k], ref[k]) < 1e-12, k
    assert _rel(out["dk_vs"], ref["dk_vs"]) < 1e-12
