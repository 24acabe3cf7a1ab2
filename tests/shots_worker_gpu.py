"""One rank of the sharded-engine check on a GPU (launched by test_shots_dist.py).

Both ranks share one GPU and exchange the shot sums over gloo (a host-side all-reduce), so
no kernel of one rank waits on the other.  Rank 0 also runs the whole survey on one engine
and writes both gradients and misfits to the .npz named on the command line.
"""
import datetime
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402
import torch  # noqa: E402
import torch.distributed as dist  # noqa: E402

from swd_b200 import configs  # noqa: E402
from swd_b200.engine import GradientEngine  # noqa: E402
from swd_b200.shots import ShardedGradient  # noqa: E402


def main(out):
    rank = int(os.environ["RANK"])
    world = int(os.environ["WORLD_SIZE"])
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(0)
    s = configs.tiny(nt=400, ns=5)
    sg = ShardedGradient(s, world, rank, device=0)
    sg.set_observed_from_model(s.vp_true, s.vs_true)
    d_vp = torch.from_numpy(np.ascontiguousarray(s.vp.T)).cuda()
    d_vs = torch.from_numpy(np.ascontiguousarray(s.vs.T)).cuda()
    d_dk = torch.zeros((s.nx, s.nz), dtype=torch.float64, device="cuda")
    mis = sg.gradient_device(d_vp, d_vs, d_dk)
    dk = d_dk.cpu().numpy().T
    if rank == 0:
        with GradientEngine(s) as e:
            cr, cl = e.observed_curves(s.vp_true, s.vs_true)
            e.set_observed(cr, cl)
            ref = e.gradient(s.vp, s.vs)
        np.savez(out, dk=dk, mis=mis, ref_dk=ref["dk_vs"], ref_mis=ref["residual"], shots=sg.shots)
    dist.barrier()
    sg.close()
    dist.destroy_process_group()


if __name__ == "__main__":
    main(sys.argv[1])
