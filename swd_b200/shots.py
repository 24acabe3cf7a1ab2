"""Shots sharded over ranks: the parfor over shots of SWD.m:171-194 spread across GPUs.

Every rank runs its share of the survey's shots through its own GradientEngine.  The
gradient needs one exchange: the FP64 shot sums of g_cl, g_cm and g_illum (SWD.m:193)
and the right-side misfit sum and count (SWD.m:196) are summed over ranks, after which
each rank assembles the same smoothed Vs gradient (SWD.m:199-201).  Nothing else
crosses ranks: models, materials and Radon tables are built on every rank.

The exchange goes through torch.distributed (NCCL on GPUs, gloo on CPUs); on GPUs it is
issued on the engine's stream so that it follows the shot sums without a host sync.
"""
from __future__ import annotations

import dataclasses

import numpy as np


def shard(ns, world, rank):
    """1-based shot numbers of rank `rank`: round robin, so every rank gets shots from the whole
    line and the counts differ by at most one (all shots of a survey cost the same)."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside 0..{world - 1}")
    return np.arange(rank + 1, ns + 1, world, dtype=np.int32)


def subset(survey, shots):
    """The survey restricted to `shots` (1-based numbers in `survey`), keeping their numbers."""
    shots = np.asarray(shots, np.int32)
    base = np.asarray(survey.shot_no, np.int32) if survey.shot_no is not None else np.arange(
        1, survey.ns + 1, dtype=np.int32)
    if shots.size == 0:
        raise ValueError("a rank needs at least one shot")
    return dataclasses.replace(survey, sx=np.asarray(survey.sx)[shots - 1], shot_no=base[shots - 1],
                               ns_total=survey.ns_total or survey.ns)


def allreduce_sums(gsum, misfit, group=None):
    """Sum the shot sums (3*nz*nx float64) and [misfit sum, count] over the ranks of `group`."""
    import torch.distributed as dist
    dist.all_reduce(gsum, group=group)
    dist.all_reduce(misfit, group=group)


class ShardedGradient:
    """One rank's share of an SWD gradient over `world` ranks.

    gradient_device(d_vp, d_vs, d_dk) -> misfit: (vp, vs) and dk_vs are float64 CUDA tensors
    holding MATLAB column-major nz x nx data (tensors of shape (nx, nz)).
    """

    def __init__(self, survey, world=1, rank=0, device=0, group=None, **engine_opts):
        import torch

        from .engine import GradientEngine
        self.survey, self.world, self.rank, self.group = survey, world, rank, group
        self.shots = shard(survey.ns, world, rank)
        self.local = subset(survey, self.shots)
        self.engine = GradientEngine(self.local, device=device, **engine_opts)
        dev = torch.device("cuda", device)
        self._gsum = torch.zeros(3 * survey.nz * survey.nx, dtype=torch.float64, device=dev)
        self._mis = torch.zeros(2, dtype=torch.float64, device=dev)
        self._stream = torch.cuda.ExternalStream(self.engine.stream(), device=dev)

    @property
    def stream(self):
        return self._stream

    def set_observed_from_model(self, vp_true, vs_true):
        """Observed curves of this rank's shots from a "true" model (SWD.m:155-162)."""
        cr, cl = self.engine.observed_curves(vp_true, vs_true)
        self.engine.set_observed(cr, cl)
        return cr, cl

    def gradient_device(self, d_vp, d_vs, d_dk):
        import torch
        rsum, rcnt = self.engine.shot_sums_device(d_vp, d_vs, self._gsum)
        with torch.cuda.stream(self._stream):
            self._mis[0], self._mis[1] = rsum, rcnt
            if self.world > 1:
                allreduce_sums(self._gsum, self._mis, self.group)
        self.engine.assemble_device(self._gsum, d_dk)
        s, c = self._mis.tolist()
        return s / c if c else float("nan")

    def close(self):
        self.engine.close()
