#!/usr/bin/env python
"""Shot-gradients/s of the SWD gradient hot path on one node.

A step is one SWD gradient (SWD.m:171-201) over the batched 100 x 600 survey:
96 shots x 600 receivers, nt 8000, forward FD + dispersion spectra + picks +
SoftMax adjoint sources + adjoint FD with imaging, summed over shots and
assembled into the smoothed Vs gradient.  Inputs are seeded synthetic models.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Under torchrun the survey's shots are split round-robin over the ranks (strong
scaling: the whole job is always the same 96 shots); each rank's FP64 shot sums
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
# DRAM bytes of the FD step kernels, measured with ncu (dram__bytes_read.sum +
# dram__bytes_write.sum) on the 100x600 survey (132 x 660 padded cells), per FD schedule:
# (B per padded shot-cell of a plain launch, B per interior shot-cell that a launch writing a
# snapshot (forward) or applying the imaging condition (adjoint, by image-sum precision) adds).
# A launch-averaged figure is plain * cells + (steps per launch / nt_wf) * extra * interior
# cells.  None: that variant has no capture, and the line reports traffic null.
NCU_TRAFFIC = {2: {"fd_fwd_step": (35.05, None), "fd_adj_step": (34.99, {})},
               3: {"fd_fwd_step": (35.09, 10.89), "fd_adj_step": (35.14, {"fp32": 36.67})},
               4: {"fd_fwd_step": (36.1, 13.2), "fd_adj_step": (36.1, {"fp64": 64.8})},
               5: {"fd_fwd_step": (36.00, 11.11), "fd_adj_step": (35.99, {"fp32": 36.01})},
               6: {"fd_fwd_step": (36.40, 11.07), "fd_adj_step": (36.42, {"fp32": 36.08})}}
# Compulsory DRAM bytes of the fused one-sweep kernels: 5 state fields read + 5 written per
# shot-cell and launch (a launch advances one step, or two under schedules 3 and 5; materials
# are shared by the shots of a launch), plus per interior cell every nt_wf steps the 3-field
# snapshot write (forward) or snapshot read + image update (adjoint; FP32 or FP64 sums).
# These are the bytes roofline.achieved counts.  The reference's two-phase schedule moves
# 84 B per cell-step (velocity pass, then stress pass); that figure is reported beside it.
COMPULSORY_STATE_B = 40


def parse():
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--workload", choices=["batched-100x600", "large-400x3000"], default="batched-100x600",
                   help="batched-100x600 (96 shots, nt 8000) or large-400x3000 (240 shots, nt 20000)")
    p.add_argument("--shots", type=int, default=0, help="shots in the survey (0: the workload's; split over GPUs)")
    p.add_argument("--nt", type=int, default=0, help="time steps (0: the workload's)")
    p.add_argument("--plain-shots", type=int, default=8, help="shots timed on the one-shot-per-launch path")
    p.add_argument("--cpu-shots", type=int, default=0, help="CPU baseline sample size (0: one per host thread)")
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    p.add_argument("--no-variants", action="store_true",
                   help="skip the legs with checkpoints every 50 steps and with FP64 image sums")
    p.add_argument("--snapshot-mode", type=int, default=0, help="0 auto, 1 store snapshots, 2 checkpoint")
    p.add_argument("--ckpt", type=int, default=0,
                   help="steps between checkpoints (snapshot mode 2; 0: memory-optimal)")
    p.add_argument("--warps", type=int, default=0, help="FD kernel CTA shape (0: planner default)")
    p.add_argument("--cells", type=int, default=0)
    p.add_argument("--ring", type=int, default=0)
    p.add_argument("--chunk", type=int, default=0)
    p.add_argument("--image-precision", choices=["fp32", "fp64"], default="fp32",
                   help="per-shot imaging sums: fp32 as the reference accumulates them (default) or fp64")
    p.add_argument("--sched", type=int, default=-1,
                   help="FD schedule: 0 or 3 warp streaming, two steps per launch; 1 one barrier per row; "
                        "2 warp streaming, one step; 4 two barriers per row; 5 as 3 with two shots per warp; "
                        "6 as 3 with two columns per lane (-1: autotuned)")
    p.add_argument("--serve", type=int, default=0,
                   help="served request stream: number of requests (0: run the gradient bench instead)")
    p.add_argument("--rate", type=float, default=2.0, help="served stream: Poisson arrival rate, requests/s")
    p.add_argument("--inflight", type=int, default=4, help="served stream: requests on the GPU at once")
    p.add_argument("--surveys", type=int, default=16, help="served stream: distinct surveys (engine keys)")
    p.add_argument("--radon", action="store_true",
                   help="Radon contraction precision study (200 f x 400 v x 600 offsets x 96 shots)")
    p.add_argument("--precision", action="store_true",
                   help="FP32 engine vs the full-FP64 per-shot path: seismograms, spectra, picks, gradient, misfit")
    p.add_argument("--invert", type=int, default=0,
                   help="SWD inversion iterations (gradient + line search) on the batched 100x600 survey")
    p.add_argument("--invert-plain", action="store_true",
                   help="run the inversion on the plain one-shot-per-launch path (no CUDA graphs) instead")
    p.add_argument("--plain-sample", type=int, default=8,
                   help="served stream: requests re-run serially on the plain path for the comparison")
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
    if args.workload == "large-400x3000":
        return configs.large_c5(ns=args.shots, nt=args.nt)
    return configs.batched_c2(ns=args.shots, nt=args.nt)


def workload_config(s, extra=None):
    c = {"workload": f"{s.name}: nz={s.nz} nx={s.nx} dx={s.dx} nbc={s.nbc} nt={s.nt} dt={s.dt} "
                     f"{s.ns} shots x {s.ng} receivers, Ricker f0={s.f0}, Radon {s.fmin:g}-{s.fmax:g} Hz "
                     f"df={s.df:g}, {s.vmin:g}-{s.vmax:g} m/s step {s.dv:g}, offset {s.offset}",
         "shots": s.ns, "grid_padded": [s.nzbc, s.nxbc], "nt": s.nt, "nt_wf": s.nt_wf,
         "l2": "inputs larger than L2 (state + snapshots >> 126 MB); no flush needed"}
    if extra:
        c.update(extra)
    return c


def variant_legs(s, info, cr0_r, cr0_l, dev, steps):
    """The survey's stated configuration variants, on the same kernels and shape as the main line,
    timed like `value` (inputs resident on the device, CUDA events on the engine's stream, one
    warm-up step that captures the graphs): checkpoints every 50 steps with the adjoint
    recomputing each segment, and FP64 per-shot image sums (the FP64 accumulation over time
    steps) in the main line's adjoint mode."""
    import torch

    from swd_b200.engine import GradientEngine
    shape = {k: info[k] for k in ("fd_schedule", "warps", "cells", "ring_fwd", "ring_adj")}
    shape["chunk_rows"] = info["chunk_rows"]
    legs = {"checkpoint_every_50_steps": {"snapshot_mode": 2, "ckpt_interval": 50},
            "fp64_image_sums": {"snapshot_mode": info["mode"], "image_precision": "fp64"}}
    d_vp = torch.from_numpy(np.ascontiguousarray(s.vp.T)).to(dev)
    d_vs = torch.from_numpy(np.ascontiguousarray(s.vs.T)).to(dev)
    d_dk = torch.zeros((s.nx, s.nz), dtype=torch.float64, device=dev)
    out = {}
    for name, kw in legs.items():
        with GradientEngine(s, device=dev.index, **shape, **kw) as e:
            e.set_observed(cr0_r, cr0_l)
            e.gradient_device(d_vp, d_vs, d_dk)
            st = torch.cuda.ExternalStream(e.stream(), device=dev)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(steps):
                e.gradient_device(d_vp, d_vs, d_dk)
            e1.record(st)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / steps
            out[name] = {"value": s.ns / (ms / 1e3), "unit": UNIT, "ms_per_step": ms, "steps": steps,
                         "adjoint": {1: "stored strain snapshots", 2: "checkpoint+recompute"}[e.info["mode"]],
                         "ckpt_interval": e.info["ckpt_interval"], "image_sums": kw.get("image_precision", "fp32")}
    return out


# ------------------------------------------------------------------ CPU baseline (the reference's CPU path)

def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline(s, n_shots=0, fd=None):
    """Time the reference's CPU path on a bounded sample: one full shot-gradient per host thread
    (SWD.m's parfor over shots).  The FD steps run the reference's own MEX sources built into
    oracle/_ref (kind 'reference') when they are here, else the restated C++ oracle ('port');
    the Radon / pick / SoftMax steps are the oracle's numpy restatement of the .m files either
    way (MATLAB is not available to run them)."""
    import psutil
    from concurrent.futures import ThreadPoolExecutor

    from oracle import swd_oracle as O
    from oracle import swd_ref
    if fd is None:
        fd = "reference" if swd_ref.available() else "oracle"
    cores = os.cpu_count() or 1
    mem_gb = psutil.virtual_memory().available / 2**30
    per_shot_gb = 4 * s.nz * s.nx * (s.nt // s.nt_wf) * 4 / 2**30 * 1.3 + 0.5
    n = n_shots or max(1, min(cores, int(mem_gb * 0.6 / per_shot_gb)))
    cr0 = np.ones((s.npair, s.ns))
    shots = [1 + (i * max(1, s.ns // n)) % s.ns for i in range(n)]
    t0 = time.perf_counter()
    with ThreadPoolExecutor(n) as ex:
        list(ex.map(lambda i: O.shot_gradient(s, i, s.vs, cr0, cr0, fd=fd), shots))
    dt = time.perf_counter() - t0
    what = ("FD on the reference's MEX sources (oracle/_ref)" if fd == "reference" else
            "FD on the restated C++ oracle")
    return {"value": n / dt, "unit": UNIT, "cores": n, "kind": "reference" if fd == "reference" else "port",
            "cpu_model": cpu_model(), "host_threads": cores,
            "sample": f"{n} full shot-gradients of the {s.nz}x{s.nx} survey (nt {s.nt}), one per host thread, "
                      f"{dt:.1f} s wall on {cores} host threads; {what}, Radon/pick/SoftMax on the numpy "
                      f"restatement of the .m files"}


def run_reference(args):
    """--impl reference: the reference's CPU path (its FD MEX sources built unmodified in
    oracle/_ref, the .m steps restated in numpy; MATLAB itself cannot run here)."""
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
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(s),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": info["cores"], "kind": info["kind"],
                             "cpu_model": info["cpu_model"], "sample": info["sample"]},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ our arm

def run_serve(args):
    """Served request stream on one GPU: Poisson arrivals of gradient and misfit requests over
    surveys of different grid sizes, shot counts and nt; p50/p99 latency and throughput, next to
    the same kind of requests run one at a time on the plain one-shot-per-launch path."""
    from swd_b200 import configs
    from swd_b200.engine import GradientEngine
    from swd_b200.serve import Server
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    surveys = configs.served_surveys(args.surveys)
    stream = configs.served_stream(args.serve, len(surveys), args.rate)
    cr0 = [configs.smooth_curve(s, i) for i, s in enumerate(surveys)]

    def inputs(k, sc):
        s = surveys[k]
        vs = s.vs * sc
        return s, s.vp_ratio * vs, vs

    # warm: library load and one small request
    with Server(max_inflight=1) as srv:
        s, vp, vs = inputs(0, 1.0)
        srv.wait(srv.submit(s, vp, vs, cr0[0], cr0[0], kind="misfit"))
    with Server(max_inflight=args.inflight) as srv, ClockSampler(0) as clk:
        t0 = time.perf_counter()
        ids = []
        for t, k, kind, sc in stream:
            lag = t0 + t - time.perf_counter()
            if lag > 0:
                time.sleep(lag)
            s, vp, vs = inputs(k, sc)
            ids.append(srv.submit(s, vp, vs, cr0[k], cr0[k], kind=kind, key=k + 1))
        results = [srv.wait(i) for i in ids]
        wall = time.perf_counter() - t0
        st = srv.stats()
    lat = np.array([r["total_ms"] for r in results])
    shots = sum(surveys[k].ns for _, k, kind, _ in stream if kind == "gradient")
    # the plain path, one request at a time, on every (n/sample)-th request of the same stream
    step = max(1, len(stream) // max(1, args.plain_sample))
    sample = stream[::step][: args.plain_sample]
    tp = time.perf_counter()
    for _, k, kind, sc in sample:
        s, vp, vs = inputs(k, sc)
        with GradientEngine(s, max_batch=1, use_graphs=False) as e:
            e.set_observed(cr0[k], cr0[k])
            (e.gradient if kind == "gradient" else e.misfit)(vp, vs)
    tp = time.perf_counter() - tp
    line = {"metric": "served requests/s", "value": len(stream) / wall, "unit": "requests/s", "n_gpus": 1,
            "higher_is_better": True, "dtype": "f32", "data": "synthetic (seeded layered models + checkerboard)",
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                           "mean": float(lat.mean()), "max": float(lat.max())},
            "shot_gradients_per_s": shots / wall,
            "config": {"workload": f"{len(stream)} requests (gradient or line-search misfit), Poisson arrivals at "
                                   f"{args.rate:g}/s over {len(surveys)} surveys: grids 60x200..300x1200 "
                                   f"(log-uniform), 8-64 shots, nt 3000-10000, dx 0.5, nbc 30, dt 5e-5",
                       "max_inflight": args.inflight, "arrival_span_s": stream[-1][0]},
            "server": {k: st[k] for k in ("admitted", "completed", "waits_for_memory", "peak_inflight",
                                          "peak_bytes", "budget")},
            "engine_reuse": sum(r["reused_engine"] for r in results),
            "plain_serial": {"requests": len(sample), "seconds": tp, "value": len(sample) / tp, "unit": "requests/s",
                             "how": "same requests (every n-th of the stream), one at a time, one shot per launch, "
                                    "no CUDA graphs"},
            "clocks": clk.summary()}
    line["served_over_plain"] = line["value"] / line["plain_serial"]["value"]
    print(json.dumps(line), flush=True)
    return 0


def radon_inputs(nf=200, npv=400, nx=600, ns=96, nt=1000, dt=1e-3, seed=11):
    """Axes of the precision study and complex64 spectra of seeded band-limited Gaussian traces:
    white noise band-passed to 3-80 Hz in the FFT domain, then a direct DFT at the nf frequencies."""
    rng = np.random.default_rng(seed)
    freq = np.linspace(3.0, 80.0, nf)
    vel = np.linspace(80.0, 1200.0, npv)
    off = np.arange(nx) * 0.5
    u = rng.standard_normal((ns * nx, nt)).astype(np.float32)
    fu = np.fft.rfft(u, axis=1)
    fr = np.fft.rfftfreq(nt, dt)
    fu[:, (fr < 3.0) | (fr > 80.0)] = 0
    u = np.fft.irfft(fu, nt, axis=1).astype(np.float32)
    e = np.exp(-2j * np.pi * np.outer(np.arange(nt) * dt, freq)).astype(np.complex64)  # [t, f]
    spec = (u @ e).reshape(ns, nx, nf).transpose(0, 2, 1)  # [s, f, x]
    return freq, vel, off, np.ascontiguousarray(spec.astype(np.complex64).astype(np.complex128))


def run_radon(args):
    """Radon contraction in FP64, FP32 (CUDA cores) and split-BF16 (tcgen05): time per launch,
    GFLOP/s, tensor-pipe FLOP/s against the measured bf16 peak, and the error of the spectrum,
    its column-normalised amplitude and its argmax picks against the FP64 path."""
    import torch

    from swd_b200 import kernel_launches
    from swd_b200.contract import Contraction
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    freq, vel, off, spec = radon_inputs()
    ns = spec.shape[0]
    d_spec = torch.from_numpy(spec).cuda()
    peaks_j = {}
    pf = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pf):
        peaks_j = json.load(open(pf))
    out, ref = {}, None
    for prec in ("fp64", "fp32", "bf16x2", "bf16x3"):
        with Contraction(freq, vel, off, ns, prec) as c:
            d_mm = torch.zeros(c.shape_out, dtype=torch.complex128, device="cuda")
            st = torch.cuda.current_stream()
            for _ in range(max(3, args.warmup)):
                c.run(d_spec, d_mm, st)
            torch.cuda.synchronize()
            reps = max(5, args.steps)
            l0 = kernel_launches()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(reps):
                c.run(d_spec, d_mm, st)
            e1.record(st)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / reps
            useful, issued = c.flops()
            timed_out = c.timed_out()
            mm = d_mm.cpu().numpy()
        r = {"ms": ms, "gflops": useful / ms / 1e6, "launches_per_run": (kernel_launches() - l0) / reps,
             "timed_out": timed_out}
        if prec.startswith("bf16"):
            tf = issued / ms / 1e9
            pk = peaks_j.get("bf16_tflops", 1590.0)
            r["tensor"] = {"achieved": tf, "peak": pk, "unit": "TFLOP/s", "frac": tf / pk,
                           "peak_source": "measured bf16_tflops" if peaks_j else "fallback 1590"}
        if ref is None:
            ref = mm
        else:
            amp, aref = np.abs(mm), np.abs(ref)
            nmax, rmax = amp / amp.max(axis=2, keepdims=True), aref / aref.max(axis=2, keepdims=True)
            r["rel_l2_mm"] = float(np.linalg.norm(mm - ref) / np.linalg.norm(ref))
            r["rel_l2_spectrum"] = float(np.linalg.norm(nmax - rmax) / np.linalg.norm(rmax))
            r["pick_agreement"] = float(np.mean(amp.argmax(axis=2) == aref.argmax(axis=2)))
        out[prec] = r
    line = {"metric": "Radon contraction GFLOP/s (split-BF16 tcgen05)", "value": out["bf16x2"]["gflops"],
            "unit": "GFLOP/s", "n_gpus": 1, "higher_is_better": True, "dtype": "bf16x2 (FP32 accumulate)",
            "data": "synthetic: complex64 spectra of seeded band-limited Gaussian traces",
            "config": {"workload": "200 frequencies 3-80 Hz x 400 velocities 80-1200 m/s x 600 offsets 0.5 m x "
                                   "96 shots", "useful_gflop": 8 * 200 * 400 * 600 * 96 / 1e9},
            "precisions": out}
    print(json.dumps(line), flush=True)
    return 0


def run_precision(args):
    """Relative errors of the FP32 path against the full-FP64 path on the same inputs.

    FP32 path: the batched engine (FP32 FD with FP64 image accumulation, FP64 spectra, picks
    and SoftMax) and, for seismograms and spectra, the FP32 MEX-convention calls per shot.
    FP64 path: SWD.m's shot loop on the double MEX pair (swd_b200.swd_loop, single=False).
    Both use the same observed curves (the FP32 engine's picks of the true model)."""
    from swd_b200 import configs, shots, swd_loop
    from swd_b200.engine import GradientEngine
    if int(os.environ.get("RANK", "0")) != 0:
        return 0

    def rel(a, b):
        a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
        return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))

    cases = (("plain-30x120, 12 shots, nt 6000", configs.plain_c1()),
             ("batched-100x600, shots 1/25/49/73 of 96, nt 8000",
              shots.subset(configs.batched_c2(), [1, 25, 49, 73])))
    out = {}
    for name, s in cases:
        with GradientEngine(s) as e:
            cr0_r, cr0_l = e.observed_curves(s.vp_true, s.vs_true)
            e.set_observed(cr0_r, cr0_l)
            g32 = e.gradient(s.vp, s.vs)
        with GradientEngine(s, radon_precision="bf16x2") as e:  # FP32 FD + split-BF16 Radon
            e.set_observed(cr0_r, cr0_l)
            gbf = e.gradient(s.vp, s.vs)
        g64 = swd_loop.gradient(s, s.vs, cr0_r, cr0_l, single=False, keep_shots=True)
        seis, spec = [], []
        for is_ in range(1, s.ns + 1):
            sw32, _ = swd_loop._seismogram(s, is_, s.vs, True)
            p64 = g64["per_shot"][is_ - 1]
            seis.append(rel(sw32, p64["seismo_w"]))
            sp32 = swd_loop.spectra(s, sw32, is_)
            for side in ("r", "l"):
                if side in sp32:
                    spec.append(rel(sp32[side][0], p64["ml_" + side]))
        picks32 = np.concatenate([g32["cr_pre_r"].ravel(), g32["cr_pre_l"].ravel()])
        picks64 = np.concatenate([g64["cr_pre_r"].ravel(), g64["cr_pre_l"].ravel()])
        out[name] = {
            "seismogram_rel_l2": {"max": max(seis), "median": float(np.median(seis))},
            "spectrum_rel_l2": {"max": max(spec), "median": float(np.median(spec))},
            "picks": {"identical_fraction": float(np.mean(picks32 == picks64)),
                      "max_abs_diff_m_s": float(np.max(np.abs(picks32 - picks64)))},
            "gradient_rel_l2": {k: rel(g32[k], g64[k]) for k in ("dk_vs", "g_cl", "g_cm", "g_illum")},
            "misfit_rel": abs(g32["residual"] - g64["residual"]) / abs(g64["residual"]),
        }
        pbf = np.concatenate([gbf["cr_pre_r"].ravel(), gbf["cr_pre_l"].ravel()])
        out[name]["with_split_bf16_radon"] = {
            "picks_identical_fraction": float(np.mean(pbf == picks64)),
            "picks_max_abs_diff_m_s": float(np.max(np.abs(pbf - picks64))),
            "gradient_rel_l2": rel(gbf["dk_vs"], g64["dk_vs"]),
            "misfit_rel": abs(gbf["residual"] - g64["residual"]) / abs(g64["residual"])}
    line = {"metric": "FP32 path relative error vs full FP64", "value": max(v["gradient_rel_l2"]["dk_vs"]
                                                                           for v in out.values()),
            "unit": "relative L2 of the Vs gradient (worst case)", "higher_is_better": False, "n_gpus": 1,
            "dtype": "f32 FD, f64 accumulation / spectra / SoftMax", "data": "synthetic", "cases": out}
    print(json.dumps(line), flush=True)
    return 0


def run_invert(args):
    """SWD.m's inversion loop on the engine: iterations/hour, misfit per iteration and the
    forward/gradient passes each iteration took (the starting model is linear in depth
    between the true model's extremes, SWD.m:27-30)."""
    import torch

    from swd_b200 import configs
    from swd_b200.invert import Inversion
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    s = survey(args)
    vs0 = np.repeat(np.linspace(np.min(s.vs_true), np.max(s.vs_true), s.nz)[:, None], s.nx, 1)
    opts = {"max_batch": 1, "use_graphs": False} if args.invert_plain else {"autotune": True}
    inv = Inversion(s, vs0, s.vs_true, **opts)
    inv.run(1)  # warm-up: engine, graphs, observed curves
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    hist = inv.run(args.invert)
    dt = time.perf_counter() - t0
    err0 = float(np.sqrt(np.mean((vs0 - s.vs_true) ** 2)))
    err1 = float(np.sqrt(np.mean((inv.vs - s.vs_true) ** 2)))
    inv.close()
    line = {"metric": "SWD iterations/hour", "value": len(hist[1:]) / dt * 3600 if len(hist) > 1 else None,
            "unit": "iterations/hour", "n_gpus": 1, "higher_is_better": True, "dtype": "f32",
            "data": "synthetic (seeded layered model + Gaussian anomaly)",
            "config": workload_config(s, {"iterations_timed": len(hist) - 1,
                                          "path": "plain: one shot per launch, no CUDA graphs" if args.invert_plain
                                          else "batched engine, CUDA graphs, autotuned"}),
            "seconds_per_iteration": dt / max(1, len(hist) - 1),
            "residual": [h.residual for h in hist], "accepted_misfit": [h.res0 for h in hist],
            "misfit_passes": [h.misfit_passes for h in hist], "offset": [h.offset for h in hist],
            "vs_rms_error_m_s": {"start": err0, "end": err1}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if not args.shots:
        args.shots = 240 if args.workload == "large-400x3000" else 96
    if not args.nt:
        args.nt = 20000 if args.workload == "large-400x3000" else 8000
    if args.invert:
        return run_invert(args)
    if args.precision:
        return run_precision(args)
    if args.impl == "reference":
        return run_reference(args)
    if args.serve:
        return run_serve(args)
    if args.radon:
        return run_radon(args)
    import torch
    import torch.distributed as dist

    import swd_b200 as S
    from swd_b200.engine import GradientEngine
    from swd_b200.shots import ShardedGradient

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    s = survey(args)
    # this rank's share of the survey's shots (all of them at N=1)
    # the engine times its FD kernel variants on this survey unless a shape is given
    tune = not (args.warps or args.cells or args.ring or args.chunk or args.sched >= 0)
    sg = ShardedGradient(s, world, rank, device=local, snapshot_mode=args.snapshot_mode,
                         ckpt_interval=args.ckpt, warps=args.warps, cells=args.cells, ring_fwd=args.ring,
                         ring_adj=args.ring, chunk_rows=args.chunk, autotune=tune,
                         fd_schedule=max(args.sched, 0), image_precision=args.image_precision)
    eng = sg.engine
    info = eng.info
    # observed curves of the "true" model (setup, SWD.m:155-162), then resident inputs
    cr0_r, cr0_l = sg.set_observed_from_model(s.vp_true, s.vs_true)
    dev = torch.device("cuda", local)
    # MATLAB column-major nz x nx data == C-contiguous (nx, nz)
    d_vp = torch.from_numpy(np.ascontiguousarray(s.vp.T)).to(dev)
    d_vs = torch.from_numpy(np.ascontiguousarray(s.vs.T)).to(dev)
    d_dk = torch.zeros((s.nx, s.nz), dtype=torch.float64, device=dev)
    ext = sg.stream

    def step():
        return sg.gradient_device(d_vp, d_vs, d_dk)

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
    value = s.ns / (ms_step / 1e3)  # the survey's shots, over all ranks

    # e2e from pinned host memory: (vp, vs) up, gradient (+ images, picks, misfits at N=1) down.
    # N=1: the host-pointer C ABI call swd_engine_gradient; N>1: copies around the sharded step.
    vp_h = torch.empty((s.nx, s.nz), dtype=torch.float64, pin_memory=True)
    vs_h = torch.empty((s.nx, s.nz), dtype=torch.float64, pin_memory=True)
    dk_h = torch.empty((s.nx, s.nz), dtype=torch.float64, pin_memory=True)
    vp_h.numpy()[:] = s.vp.T
    vs_h.numpy()[:] = s.vs.T

    def e2e_step():
        if world == 1:
            eng.gradient(vp_h.numpy().T, vs_h.numpy().T)
            return
        with torch.cuda.stream(ext):
            d_vp.copy_(vp_h, non_blocking=True)
            d_vs.copy_(vs_h, non_blocking=True)
        sg.gradient_device(d_vp, d_vs, d_dk)
        dk_h.copy_(d_dk)

    if args.steps < 1:
        e2e_step()  # warm (the timed steps already captured the engine's graphs otherwise)
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    ne2e = max(1, min(args.steps, 3))
    for _ in range(ne2e):
        e2e_step()
    e2e_s = (time.perf_counter() - t0) / ne2e
    if world > 1:
        t = torch.tensor([e2e_s], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    h2d = 2 * s.nz * s.nx * 8
    d2h = (4 * s.nz * s.nx * 8 + 2 * s.ns * 8 + 2 * info["npair"] * s.ns * 8) if world == 1 else s.nz * s.nx * 8 + 16

    # roofline of the FD step kernels from the per-phase CUDA events of the timed steps
    fwd_ms = statistics.mean(p[0] for p in phases)
    adj_ms = statistics.mean(p[2] for p in phases)
    spec_ms = statistics.mean(p[1] for p in phases)
    nloc = sg.local.ns  # shots of this rank: one FD launch steps all of them
    cells = s.nzbc * s.nxbc * nloc
    inner = s.nz * s.nx * nloc
    # the reference's two-phase schedule per time step of every shot: 84 B per padded cell-step,
    # plus 16 B snapshot write (forward) or 16 B snapshot read + 24 B FP32 image update
    # (adjoint) per interior cell every nt_wf steps; times the steps per launch
    spl = 2 if info["fd_schedule"] in (3, 5, 6) else 1  # time steps per launch
    fwd_bytes = spl * (cells * 84 + inner * 16 / s.nt_wf)
    img_rmw = 24 if args.image_precision == "fp32" else 48  # 3 image sums read and written
    adj_bytes = spl * (cells * 84 + inner * (16 + 24) / s.nt_wf)  # the reference's FP32 image sums
    # compulsory bytes of a launch: the state once in and out, the materials once (one float4 per
    # cell, shared by the shots), 3 snapshot fields written (forward) or read with the 3 image
    # sums read and written (adjoint) per interior cell every nt_wf steps
    mat = s.nzbc * s.nxbc * 16
    snaps = info["mode"] == 1  # checkpoint mode: the forward phase writes no snapshots
    fwd_comp = cells * COMPULSORY_STATE_B + mat + (spl * inner * 12 / s.nt_wf if snaps else 0)
    adj_comp = cells * COMPULSORY_STATE_B + mat + spl * inner * (12 + img_rmw) / s.nt_wf
    fwd_launch_ms = fwd_ms / s.nt * spl
    # checkpoint mode: the adjoint phase also re-runs the forward steps segment by segment
    adj_launch_ms = ((adj_ms - fwd_ms) if info["mode"] == 2 else adj_ms) / (s.nt - 1) * spl
    peak, peak_kind = peaks()

    def roof(name, ref_bytes, comp, launch_ms):
        # achieved: the compulsory bytes of one launch (state once in and out, materials,
        # snapshot / image terms) over its average CUDA-event time
        ach = comp / (launch_ms / 1e3) / 1e9
        plain, extra = NCU_TRAFFIC.get(info["fd_schedule"], {}).get(name, (None, None))
        if name == "fd_adj_step":
            extra = (extra or {}).get(args.image_precision)
        elif not snaps:
            extra = 0.0
        tr = plain * cells + spl / s.nt_wf * extra * inner if plain is not None and extra is not None else None
        return {"kernel": name, "bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs, copy kernel)" if peak_kind == "measured"
                else "fallback 6650 GB/s",
                "traffic": tr,
                "traffic_source": (f"ncu dram__bytes_read.sum + dram__bytes_write.sum of FD schedule "
                                   f"{info['fd_schedule']}: plain launches and the snapshot / imaging variants, "
                                   "averaged over the launches of the phase") if tr else
                f"no ncu capture of every variant of FD schedule {info['fd_schedule']} with "
                f"{args.image_precision} image sums",
                "steps_per_launch": spl, "algorithmic_bytes_per_launch": comp,
                "algorithmic_bytes": "compulsory: 40 B per shot-cell per launch (5 state fields in and out) + "
                                     "snapshot write / snapshot read + image update per interior cell every "
                                     "nt_wf steps",
                "avg_launch_ms": launch_ms,
                "reference_schedule_bytes_per_launch": ref_bytes,
                "frac_reference_schedule": ref_bytes / (launch_ms / 1e3) / 1e9 / peak}

    rf = roof("fd_fwd_step", fwd_bytes, fwd_comp, fwd_launch_ms)
    ra = roof("fd_adj_step", adj_bytes, adj_comp, adj_launch_ms)
    dominant, other = (ra, rf) if adj_ms >= fwd_ms else (rf, ra)

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded layered model + Gaussian anomaly)",
            "config": workload_config(s),
            "engine": {"adjoint": {1: "stored strain snapshots", 2: "checkpoint+recompute"}[info["mode"]],
                       "ckpt_interval": info.get("ckpt_interval"), "batch": info["batch"], "engine_bytes": info["bytes"],
                       "fd_variant": {k: info[k] for k in ("fd_schedule", "warps", "cells", "ring_fwd", "ring_adj",
                                                           "chunk_rows")} | {"autotuned": tune},
                       "image_sums": args.image_precision,
                       "parallelism": f"{s.ns} shots split round-robin over {world} GPU(s), one FP64 all-reduce "
                                      f"of the shot sums per step", "shots_this_rank": nloc},
            "e2e": {"value": s.ns / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "roofline": dominant, "roofline_other": other,
            "phase_ms": {"forward": fwd_ms, "spectra_picks_adjoint_sources": spec_ms, "adjoint": adj_ms},
            "clocks": clk.summary()}

    # the plain one-shot-per-launch GPU path on a few shots (rank 0 only, N=1 only)
    if world == 1 and args.plain_shots > 0:
        from swd_b200 import shots
        ps = shots.subset(s, np.arange(1, args.plain_shots + 1))  # shots 1..k, numbered as in the survey
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
    sg.close()
    if world == 1 and not args.no_variants and args.workload == "batched-100x600":
        line["variants"] = variant_legs(s, info, cr0_r, cr0_l, dev, max(1, min(args.steps, 2)))
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
