"""Shots sharded over ranks (swd_b200.shots): partition rules and a 2-rank gloo reduction on CPU."""
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

from swd_b200 import configs, shots

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("ns,world", [(96, 1), (96, 2), (96, 8), (5, 2), (7, 3), (3, 4)])
def test_shard_partitions_the_shots(ns, world):
    if ns < world:
        with pytest.raises(ValueError):
            shots.subset(configs.tiny(ns=ns), shots.shard(ns, world, world - 1))
        return
    parts = [shots.shard(ns, world, r) for r in range(world)]
    allv = np.concatenate(parts)
    assert sorted(allv.tolist()) == list(range(1, ns + 1))
    assert max(p.size for p in parts) - min(p.size for p in parts) <= 1


def test_subset_keeps_global_shot_numbers():
    s = configs.batched_c2()
    a = shots.subset(s, shots.shard(96, 4, 1))
    assert a.ns == 24 and a.ns_total == 96
    assert a.shot_no.tolist() == list(range(2, 97, 4))
    assert np.array_equal(a.sx, s.sx[a.shot_no - 1])
    b = shots.subset(a, [2, 3])  # a subset of a subset keeps the original numbers
    assert b.shot_no.tolist() == [6, 10] and b.ns_total == 96 and b.sx.tolist() == s.sx[[5, 9]].tolist()


def _free_port():
    with socket.socket() as k:
        k.bind(("127.0.0.1", 0))
        return k.getsockname()[1]


def test_two_gloo_ranks_reduce_to_the_single_process_gradient(O, tmp_path):
    out = str(tmp_path / "r0.npz")
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()), WORLD_SIZE="2")
    procs = [subprocess.Popen([sys.executable, os.path.join(HERE, "shots_worker.py"), out],
                              env=dict(env, RANK=str(r), LOCAL_RANK=str(r)), stdout=subprocess.PIPE,
                              stderr=subprocess.STDOUT) for r in range(2)]
    try:
        logs = [p.communicate(timeout=300)[0].decode() for p in procs]
    finally:
        for p in procs:
            if p.poll() is None:
                p.kill()
    assert all(p.returncode == 0 for p in procs), logs
    r = np.load(out)
    s = configs.tiny(ns=5)
    cr0 = np.ones((s.npair, s.ns))
    ref = O.gradient(s, s.vs, cr0, cr0)
    n = s.nz * s.nx
    for k, key in enumerate(("g_cl", "g_cm", "g_illum")):
        np.testing.assert_allclose(r["gsum"][k * n:(k + 1) * n], ref[key].reshape(-1), rtol=1e-12, atol=0)
    assert r["mis"][0] / r["mis"][1] == pytest.approx(ref["residual"], rel=1e-12)
    g = r["gsum"].reshape(3, s.nz, s.nx)
    dk = O.assemble(s.vs, g[0], g[1], g[2], s.smooth_z, s.smooth_x)
    np.testing.assert_allclose(dk, ref["dk_vs"], rtol=1e-10, atol=1e-300)


@pytest.mark.gpu
def test_two_ranks_of_sharded_engines_reduce_to_the_one_engine_gradient(tmp_path):
    """The GPU path of the shard/reduce logic: two ranks with their own engines and shot shares
    on one GPU, the shot sums all-reduced over gloo, against one engine over all shots."""
    out = str(tmp_path / "g0.npz")
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()), WORLD_SIZE="2")
    procs = [subprocess.Popen([sys.executable, os.path.join(HERE, "shots_worker_gpu.py"), out],
                              env=dict(env, RANK=str(r), LOCAL_RANK=str(r)), stdout=subprocess.PIPE,
                              stderr=subprocess.STDOUT) for r in range(2)]
    try:
        logs = [p.communicate(timeout=300)[0].decode() for p in procs]
    finally:
        for p in procs:
            if p.poll() is None:
                p.kill()
    assert all(p.returncode == 0 for p in procs), logs
    r = np.load(out)
    assert r["shots"].tolist() == [1, 3, 5]
    a, b = r["dk"], r["ref_dk"]
    assert np.array_equal(np.isnan(a), np.isnan(b))
    m = ~np.isnan(b)
    assert np.linalg.norm(a[m] - b[m]) / np.linalg.norm(b[m]) < 1e-12
    assert float(r["mis"]) == pytest.approx(float(r["ref_mis"]), rel=1e-12)
