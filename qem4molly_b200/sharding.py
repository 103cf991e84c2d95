"""One QEM system sharded over the ranks of a torch.distributed group.

Each rank holds the whole system (positions, charges, the same k-set) and
evaluates its share through the library (Engine.set_shard): a contiguous
block of the pair list and a contiguous block of the k-set rows, weighted
as part of the full set; rank 0 adds the per-particle terms (self image,
walls, k = 0).  The one exchange step is a sum all-reduce of the N x 3
forces (and the energy): NCCL over NVLink between GPUs, gloo on CPU.

    eng = Engine(...); eng.sample_kset(seed, P)     # same seed on every rank
    sh = ShardedEngine(eng)                         # uses the default group
    E = sh.forces_device(xyz, q, F, energy=True)    # F, E: the full result
"""
from __future__ import annotations

from . import _lib as L


def shard_bounds(n: int, rank: int, world: int) -> tuple[int, int]:
    """[lo, hi) of rank's contiguous block of n items, the split the library
    applies to the pair list and the k-set rows."""
    return (n * rank) // world, (n * (rank + 1)) // world


def kset_shard(k3, sum_K, rank, world):
    """Rows of the k-set that rank evaluates and the normaliser that keeps
    their weight sum_K / P of the full set: (rows, sum_K * rows / P)."""
    P = len(k3)
    lo, hi = shard_bounds(P, rank, world)
    return k3[lo:hi], (sum_K * (hi - lo) / P if P else 0.0)


class ShardedEngine:
    """Engine share of one system plus the all-reduce that completes it."""

    def __init__(self, engine, group=None):
        import torch.distributed as dist

        self.engine = engine
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        engine.set_shard(self.rank, self.world)

    def forces_device(self, xyz, q, F, terms=L.QEM_TERM_ALL, energy=False):
        """F (device tensor) receives the full forces; returns the full energy or None."""
        import torch
        import torch.distributed as dist

        E = self.engine.forces_device(xyz, q, F, terms=terms, energy=energy)
        dist.all_reduce(F, group=self.group)
        if energy:
            t = torch.tensor([E], dtype=torch.float64, device=F.device)
            dist.all_reduce(t, group=self.group)
            return float(t.item())
        return None
