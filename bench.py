#!/usr/bin/env python
"""Shot-gradients/s of the SWD gradient hot path on one node.

A step is one SWD gradient (SWD.m:171-201) over the batched 100 x 600 survey:
96 shots x 600 receivers, nt 8000, forward FD + dispersion spectra + picks +
SoftMax adjoint sources + adjoint FD with imaging, summed over shots and
assembled into the smoothed Vs gradient.  Inputs are seeded synthetic models.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Under torchrun every rank runs its own 96 shots (weak scaling); the shot sums
are all-reduced over NCCL before the gradient is assembled (the parfor sum of
SWD.m:193).  Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "shot-gradients/s (fwd+adj)"
UNIT = "shot-gradients/s"
# DRAM traffic per padded cell and time step of the FD step kernels, from the ncu capture
# summarised in profiles/fd_step_kernels_batched-100x600.md (dram__bytes_read.sum +
# dram__bytes_write.sum per launch / cells per launch).  None until measured.
NCU_BYTES_PER_CELL_STEP = {"fd_fwd_step": None, "fd_adj_step": None}


def parse():
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--shots", type=int, default=96, help="shots per GPU")
    p.add_argument("--nt", type=int, default=8000)
    p.add_argument("--plain-shots", type=int, default=8, help="shots timed on the one-shot-per-launch path")
    p.add_argument("--cpu-shots", type=int, default=0, help="CPU baseline sample size (0: one per host thread)")
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    p.add_argument("--snapshot-mode", type=int, default=0)
    p.add_argument("--warps", type=int, default=0, help="FD kernel CTA shape (0: planner default)")
    p.add_argument("--cells", type=int, default=0)
    p.add_argument("--ring", type=int, default=0)
    p.add_argument("--chunk", type=int, default=0)
    return p.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return d["hbm_gbs"], "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    self.rows.append([c.strip() for c in out.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in self.rows for n, v in zip(names, r[4:8]) if v.strip().lower() == "active"})
        pw = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "power_w_max": max(pw) if pw else None, "samples": len(self.rows)}


def survey(args):
    from swd_b200 import configs
    return configs.batched_c2(ns=args.shots, nt=args.nt)


def workload_config(s, extra=None):
    c = {"workload": f"batched-{s.nz}x{s.nx}: nz={s.nz} nx={s.nx} dx={s.dx} nbc={s.nbc} nt={s.nt} dt={s.dt} "
                     f"{s.ns} shots x {s.ng} receivers, Ricker f0={s.f0}, Radon {s.fmin:g}-{s.fmax:g} Hz "
                     f"df={s.df:g}, {s.vmin:g}-{s.vmax:g} m/s step {s.dv:g}, offset {s.offset}",
         "shots_per_gpu": s.ns, "grid_padded": [s.nzbc, s.nxbc], "nt": s.nt, "nt_wf": s.nt_wf,
         "l2": "inputs larger than L2 (state + snapshots >> 126 MB); no flush needed"}
    if extra:
        c.update(extra)
    return c


# ------------------------------------------------------------------ CPU baseline (the oracle port)

def cpu_baseline(s, n_shots=0):
    """Time the oracle's restated CPU path on a bounded sample: one full shot-gradient per host thread."""
    import psutil
    from concurrent.futures import ThreadPoolExecutor

    from oracle import swd_oracle as O
    cores = os.cpu_count() or 1
    mem_gb = psutil.virtual_memory().available / 2**30
    per_shot_gb = 4 * s.nz * s.nx * (s.nt // s.nt_wf) * 4 / 2**30 * 1.3 + 0.5
    n = n_shots or max(1, min(cores, int(mem_gb * 0.6 / per_shot_gb)))
    cr0 = np.ones((s.npair, s.ns))
    shots = [1 + (i * max(1, s.ns // n)) % s.ns for i in range(n)]
    t0 = time.perf_counter()
    with ThreadPoolExecutor(n) as ex:
        list(ex.map(lambda i: O.shot_gradient(s, i, s.vs, cr0, cr0), shots))
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": UNIT, "cores": n, "kind": "port",
            "sample": f"{n} full shot-gradients of the {s.nz}x{s.nx} survey (nt {s.nt}), one per host thread, "
                      f"{dt:.1f} s wall on {cores} host threads"}


def run_reference(args):
    """--impl reference: the reference's CPU path (restated C++/numpy oracle; the MATLAB MEX cannot be built)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    s = survey(args)
    from swd_b200 import configs
    warm = configs.tiny(nt=400)
    for _ in range(args.warmup):  # load libraries and warm caches on a small survey
        cpu_baseline(warm, 1)
    times = []
    info = None
    for _ in range(args.steps):
        r = cpu_baseline(s, args.cpu_shots)
        times.append(r["cores"] / r["value"])
        info = r
    v = info["cores"] / statistics.mean(times)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": statistics.mean(times) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(s, {"sample": info["sample"]}),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": info["cores"], "kind": "port",
                             "sample": info["sample"]},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ our arm

def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch
    import torch.distributed as dist

    import swd_b200 as S
    from swd_b200.engine import GradientEngine

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    s = survey(args)
    eng = GradientEngine(s, snapshot_mode=args.snapshot_mode, device=local, warps=args.warps, cells=args.cells,
                         ring_fwd=args.ring, ring_adj=args.ring, chunk_rows=args.chunk)
    info = eng.info
    # observed curves of the "true" model (setup, SWD.m:155-162), then resident inputs
    cr0_r, cr0_l = eng.observed_curves(s.vp_true, s.vs_true)
    eng.set_observed(cr0_r, cr0_l)
    dev = torch.device("cuda", local)
    # MATLAB column-major nz x nx data == C-contiguous (nx, nz)
    d_vp = torch.from_numpy(np.ascontiguousarray(s.vp.T)).to(dev)
    d_vs = torch.from_numpy(np.ascontiguousarray(s.vs.T)).to(dev)
    d_dk = torch.zeros((s.nx, s.nz), dtype=torch.float64, device=dev)
    d_gsum = torch.zeros(3 * s.nz * s.nx, dtype=torch.float64, device=dev)
    red = torch.zeros(2, dtype=torch.float64, device=dev)
    ext = torch.cuda.ExternalStream(eng.stream(), device=dev)

    def step():
        rsum, rcnt = eng.shot_sums_device(d_vp, d_vs, d_gsum)
        if world > 1:
            with torch.cuda.stream(ext):
                dist.all_reduce(d_gsum)
                red[0], red[1] = rsum, rcnt
                dist.all_reduce(red)
        eng.assemble_device(d_gsum, d_dk)

    for _ in range(args.warmup):
        step()
    eng.set_timing(True)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    launches0 = S.kernel_launches()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    phases = []
    with ClockSampler(local) as clk:
        ev0.record(ext)
        for _ in range(args.steps):
            step()
            phases.append(eng.phase_times())
        ev1.record(ext)
        torch.cuda.synchronize()
    launches = S.kernel_launches() - launches0
    ms = ev0.elapsed_time(ev1)
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    ms_step = ms / args.steps
    value = world * s.ns / (ms_step / 1e3)

    # e2e through the host-pointer C ABI from pinned host memory (inputs up, gradient + misfits down)
    vp_h = torch.empty((s.nx, s.nz), dtype=torch.float64, pin_memory=True).numpy()
    vs_h = torch.empty((s.nx, s.nz), dtype=torch.float64, pin_memory=True).numpy()
    vp_h[:] = s.vp.T
    vs_h[:] = s.vs.T
    eng.gradient(vp_h.T, vs_h.T)  # warm
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    ne2e = max(1, min(args.steps, 3))
    for _ in range(ne2e):
        out = eng.gradient(vp_h.T, vs_h.T)
    e2e_s = (time.perf_counter() - t0) / ne2e
    if world > 1:
        t = torch.tensor([e2e_s], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    h2d = 2 * s.nz * s.nx * 8
    d2h = 4 * s.nz * s.nx * 8 + 2 * s.ns * 8 + 2 * info["npair"] * s.ns * 8

    # roofline of the FD step kernels from the per-phase CUDA events of the timed steps
    fwd_ms = statistics.mean(p[0] for p in phases)
    adj_ms = statistics.mean(p[2] for p in phases)
    spec_ms = statistics.mean(p[1] for p in phases)
    cells = s.nzbc * s.nxbc * s.ns
    inner = s.nz * s.nx * s.ns
    fwd_bytes = cells * 84 + inner * 16 / s.nt_wf            # per launch (one time step of every shot)
    adj_bytes = cells * 84 + inner * (16 + 48) / s.nt_wf
    fwd_launch_ms = fwd_ms / s.nt
    adj_launch_ms = adj_ms / (s.nt - 1)
    peak, peak_kind = peaks()

    def roof(name, nbytes, launch_ms):
        ach = nbytes / (launch_ms / 1e3) / 1e9
        tr = NCU_BYTES_PER_CELL_STEP.get(name)
        return {"kernel": name, "bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else
                "fallback 6650 GB/s", "traffic": (tr * cells) if tr else None,
                "algorithmic_bytes_per_launch": nbytes, "avg_launch_ms": launch_ms}

    rf = roof("fd_fwd_step", fwd_bytes, fwd_launch_ms)
    ra = roof("fd_adj_step", adj_bytes, adj_launch_ms)
    dominant, other = (ra, rf) if adj_ms >= fwd_ms else (rf, ra)

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded layered model + Gaussian anomaly)",
            "config": workload_config(s, {"adjoint": {1: "stored strain snapshots", 2: "checkpoint+recompute"}[
                info["mode"]], "batch": info["batch"], "engine_bytes": info["bytes"],
                "parallelism": f"shots per GPU, {world} GPU(s)"}),
            "e2e": {"value": world * s.ns / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "roofline": dominant, "roofline_other": other,
            "phase_ms": {"forward": fwd_ms, "spectra_picks_adjoint_sources": spec_ms, "adjoint": adj_ms},
            "clocks": clk.summary()}

    # the plain one-shot-per-launch GPU path on a few shots (rank 0 only, N=1 only)
    if world == 1 and args.plain_shots > 0:
        from swd_b200 import configs
        ps = configs.batched_c2(ns=s.ns, nt=s.nt)
        ps.sx = ps.sx[: args.plain_shots]
        with GradientEngine(ps, max_batch=1, use_graphs=False) as pe:
            pe.set_observed(cr0_r[:, : args.plain_shots], cr0_l[:, : args.plain_shots])
            pe.gradient(ps.vp, ps.vs)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            pe.gradient(ps.vp, ps.vs)
            tp = time.perf_counter() - t0
        line["plain_gpu"] = {"value": args.plain_shots / tp, "unit": UNIT, "shots": args.plain_shots,
                             "how": "same kernels, one shot per launch, no CUDA graphs, host in/out per call"}
        line["batched_over_plain"] = line["e2e"]["value"] / line["plain_gpu"]["value"]
    eng.close()
    if world == 1 and rank == 0 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(s, args.cpu_shots)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
