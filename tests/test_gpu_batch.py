"""Batches of independent systems (qem_batch_*): batched forces equal the
per-system calls bit for bit; the graph-replayed velocity-Verlet run matches
an eager host loop over the per-system calls; the autotuner's choice keeps
the results.  Systems from the many-slab workload (N ~ U[200, 5000],
Lz ~ U[5, 20], density 0.01, gamma pairs ~ U(-0.95, 0.95)^2, P = 200)."""
import numpy as np
import pytest

from qem4molly_b200 import _lib as L
from qem4molly_b200 import workloads as W
from qem4molly_b200.api import Batch

pytestmark = pytest.mark.gpu


def _setup(n_sys, prec="fp64", seed=None):
    import torch

    cfgs = W.config4(seed=seed, n_systems=n_sys)
    engines = [W.engine_for(c, prec, seed=100 + i) for i, c in enumerate(cfgs)]
    N = [c["N"] for c in cfgs]
    dev = torch.device("cuda", 0)
    x = torch.tensor(np.concatenate([c["xyz"] for c in cfgs]), device=dev)
    q = torch.tensor(np.concatenate([c["q"] for c in cfgs]), device=dev)
    return cfgs, engines, N, x, q


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_batch_forces_equal_per_system_calls(prec):
    import torch

    cfgs, engines, N, x, q = _setup(12, prec)
    b = Batch(engines, N)
    F = torch.empty_like(x)
    b.forces(x, q, F)            # first call: synchronous sizing pass
    F.zero_()
    b.forces(x, q, F)            # asynchronous pass on the stream pool
    b.check()
    Fb = F.cpu().numpy()
    for c, e, o, n in zip(cfgs, engines, b.off, N):
        assert np.array_equal(Fb[o:o + n], e.forces(c["xyz"], c["q"]))


def test_batch_md_graph_matches_eager_loop():
    import torch

    cfgs, engines, N, x, q = _setup(6)
    rng = np.random.default_rng(9)
    v0 = rng.normal(scale=0.1, size=(sum(N), 3))
    b = Batch(engines, N)
    v = torch.tensor(v0, device=x.device)
    F = torch.empty_like(x)
    dt, steps = 1e-3, 20
    b.md(steps, dt, x, v, q, F)
    xg, vg = x.cpu().numpy(), v.cpu().numpy()
    for c, e, o, n in zip(cfgs, engines, b.off, N):
        xs, vs = c["xyz"].copy(), v0[o:o + n].copy()
        Lx, Ly, _ = c["L"]
        Fs = e.forces(xs, c["q"])
        for _ in range(steps):
            xs = xs + dt * vs + 0.5 * dt * dt * Fs
            xs[:, 0] -= Lx * np.floor(xs[:, 0] / Lx)
            xs[:, 1] -= Ly * np.floor(xs[:, 1] / Ly)
            Fn = e.forces(xs, c["q"])
            vs = vs + 0.5 * dt * (Fs + Fn)
            Fs = Fn
        assert np.allclose(xg[o:o + n], xs, rtol=0, atol=1e-9)
        assert np.allclose(vg[o:o + n], vs, rtol=0, atol=1e-9)


def test_batch_autotune_keeps_results():
    import torch

    cfgs, engines, N, x, q = _setup(16)
    b = Batch(engines, N)
    F = torch.empty_like(x)
    b.forces(x, q, F)
    ref = F.cpu().numpy().copy()
    w, ms = b.autotune(x, q, F)
    assert 1 <= w <= 16 and ms > 0
    F.zero_()
    b.forces(x, q, F)
    b.check()
    assert np.array_equal(F.cpu().numpy(), ref)
