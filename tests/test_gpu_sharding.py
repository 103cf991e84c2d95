"""Sharding one system over ranks through the library (qem_set_shard): the
shares of W ranks, evaluated one after another on one GPU, sum to the
unsharded forces and energy (FP64, to summation rounding); ShardedEngine
completes a share with an NCCL all-reduce (a one-rank group here: the test
box has one GPU)."""
import socket

import numpy as np
import pytest

from qem4molly_b200 import _lib as L
from qem4molly_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("fp32", 1e-6)])
def test_shards_sum_to_the_whole(world, prec, tol):
    cfg = W.config3(N=5000)
    cfg["walls"] = [dict(cutoff=1.0, sigma=1.0, eps=1.0, sub_pos=0.0, direction=1)]
    e = W.engine_for(cfg, prec)
    F0 = e.forces(cfg["xyz"], cfg["q"])
    F, E = e.forces(cfg["xyz"], cfg["q"], energy=True)
    Fs, Es = np.zeros_like(F), 0.0
    for r in range(world):
        e.set_shard(r, world)
        f, en = e.forces(cfg["xyz"], cfg["q"], energy=True)
        Fs += f
        Es += en
    e.set_shard(0, 1)
    assert W.rel_err(Fs, F)[0] <= tol
    assert abs(Es - E) <= tol * abs(E)
    assert np.array_equal(e.forces(cfg["xyz"], cfg["q"]), F0)  # leaving the shard restores the whole


def test_sharded_engine_all_reduce_one_rank():
    import datetime

    import torch
    import torch.distributed as dist

    from qem4molly_b200.sharding import ShardedEngine

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        cfg = W.config3(N=3000)
        e = W.engine_for(cfg, "fp64")
        Fh, Eh = e.forces(cfg["xyz"], cfg["q"], energy=True)
        sh = ShardedEngine(e)
        x = torch.tensor(cfg["xyz"], device="cuda")
        q = torch.tensor(cfg["q"], device="cuda")
        F = torch.empty_like(x)
        E = sh.forces_device(x, q, F, energy=True)
        assert np.array_equal(F.cpu().numpy(), Fh) and E == Eh
    finally:
        dist.destroy_process_group()
