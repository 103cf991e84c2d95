"""Host-side sharding of one system over ranks (qem4molly_b200.sharding),
world_size 2 on CPU with the gloo backend.

Each rank takes its block of the pair list and of the k-set rows with the
partition the library applies on a GPU (shard_bounds / kset_shard), computes
that share with the FP64 oracle standing in for the GPU kernels (pair rows,
self terms and the k = 0 term on rank 0 only), and the sum all-reduce must
give the unsharded oracle forces."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle as O
from qem4molly_b200.sharding import kset_shard, shard_bounds


def _system():
    rng = np.random.default_rng(41)
    N, Lb = 400, (60.0, 60.0, 10.0)
    xyz = np.stack([rng.random(N) * Lb[0], rng.random(N) * Lb[1], 0.5 + 9 * rng.random(N)], 1)
    q = rng.uniform(0.5, 1.5, N) * rng.choice([-1.0, 1.0], N)
    q[-1] -= q.sum()
    p = O.params(Lb, 0.1, 10.0, -0.6, 0.8)
    ms = [(1, 0), (0, 1), (1, 1), (2, -1), (-1, 2), (3, 1), (1, -3), (2, 2), (0, 3)]
    k3 = np.array([(2 * np.pi * a / Lb[0], 2 * np.pi * b / Lb[1], np.hypot(2 * np.pi * a / Lb[0], 2 * np.pi * b / Lb[1]))
                   for a, b in ms])
    return p, xyz, q, k3, 3.7


def _share(rank, world):
    p, xyz, q, k3, sK = _system()
    N = len(q)
    F = np.zeros((N, 3))
    pairs = O.pairs(p, xyz, method="brute")
    lo, hi = shard_bounds(len(pairs), rank, world)
    rows = O.pairs_eval(p, xyz, q, pairs[lo:hi])
    for (i, j), (fx, fy, fzi, _) in zip(pairs[lo:hi], rows):
        F[i] += (fx, fy, fzi)
        F[j] -= (fx, fy, fzi)  # F[j] -= F_ij (QEM_short.jl:47, the reference pair mode)
    kr, sKr = kset_shard(k3, sK, rank, world)
    F += O.F_long(p, xyz, q, kr, sKr)
    if rank == 0:
        F[:, 2] += O.self_eval(p, xyz, q, N)
    else:  # the k = 0 term belongs to rank 0
        F -= O.F_long(p, xyz, q, np.zeros((0, 3)), 0.0)
    return F


def _worker(rank, world, port, out_path):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        F = torch.tensor(_share(rank, world))
        dist.all_reduce(F)
        if rank == 0:
            np.save(out_path, F.numpy())
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_bounds_cover_exactly():
    for n in (0, 1, 7, 100, 1001):
        for world in (1, 2, 3, 8):
            spans = [shard_bounds(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans[:-1], spans[1:]))


def test_kset_shard_keeps_the_weight():
    k3 = np.arange(30.0).reshape(10, 3)
    for world in (2, 3, 4):
        parts = [kset_shard(k3, 5.0, r, world) for r in range(world)]
        assert np.array_equal(np.concatenate([p[0] for p in parts]), k3)
        for rows, s in parts:
            assert np.isclose(s / max(len(rows), 1), 0.5) or len(rows) == 0


def test_two_gloo_ranks_sum_to_the_unsharded_forces(tmp_path):
    out = str(tmp_path / "F.npy")
    mp.spawn(_worker, args=(2, _free_port(), out), nprocs=2, join=True)
    F = np.load(out)
    p, xyz, q, k3, sK = _system()
    Fref = O.short_forces(p, xyz, q) + O.F_long(p, xyz, q, k3, sK)
    assert np.linalg.norm(F - Fref) <= 1e-12 * np.linalg.norm(Fref)
