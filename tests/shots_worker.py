"""One gloo rank of the sharded shot-gradient check (launched by test_shots_dist.py).

Each rank takes its shots from swd_b200.shots.shard, computes their per-shot images and
misfits with the oracle, and sums them over the ranks with swd_b200.shots.allreduce_sums;
rank 0 writes the reduced sums to the .npz named on the command line.
"""
import datetime
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402
import torch  # noqa: E402
import torch.distributed as dist  # noqa: E402

from oracle import swd_oracle as O  # noqa: E402
from swd_b200 import configs, shots  # noqa: E402


def main(out):
    rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    s = configs.tiny(ns=5)
    cr0 = np.ones((s.npair, s.ns))
    n = s.nz * s.nx
    gsum = torch.zeros(3 * n, dtype=torch.float64)
    mis = torch.zeros(2, dtype=torch.float64)
    for is_ in shots.shard(s.ns, world, rank):
        p = O.shot_gradient(s, int(is_), s.vs, cr0, cr0)
        for k, key in enumerate(("cl", "cm", "il")):
            gsum[k * n:(k + 1) * n] += torch.from_numpy(np.ascontiguousarray(p[key]).reshape(-1))
        if not np.isnan(p["res_r"]):
            mis += torch.tensor([p["res_r"], 1.0], dtype=torch.float64)
    shots.allreduce_sums(gsum, mis)
    if rank == 0:
        np.savez(out, gsum=gsum.numpy(), mis=mis.numpy(), shots=shots.shard(s.ns, world, rank))
    dist.barrier()
    dist.destroy_process_group()


if __name__ == "__main__":
    main(sys.argv[1])
