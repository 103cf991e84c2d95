"""Force calls on device buffers or page-locked host buffers are recorded once
as a CUDA graph and replayed (qem_forces without energy): replays must give
the ordinary call's result bit for bit and follow every change the recorded
launches do not capture -- coordinates in the same buffer, a new k-set,
another output buffer, a pair list that outgrows its capacity, a non-finite
input."""
import numpy as np
import pytest

from qem4molly_b200 import _lib as L
from qem4molly_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch

    return torch.tensor(a, dtype=torch.float64, device="cuda")


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_replays_equal_the_ordinary_call(prec):
    cfg = W.config3(N=4000)
    e = W.engine_for(cfg, prec)
    ref = e.forces(cfg["xyz"], cfg["q"])           # pageable host memory: never replayed
    x, q = _dev(cfg["xyz"]), _dev(cfg["q"])
    F = _dev(np.zeros_like(cfg["xyz"]))
    launches = []
    for _ in range(4):                              # ordinary, record + replay, replay, replay
        F.fill_(float("nan"))
        e.forces_device(x, q, F)
        assert np.array_equal(F.cpu().numpy(), ref)
        launches.append(e.counts()["launches"])
    assert len(set(launches)) == 1 and launches[0] > 10  # a replay runs the recorded kernels


def test_replay_follows_coordinates_kset_and_buffers():
    import torch

    cfg = W.config3(N=4000)
    e = W.engine_for(cfg, "fp64")
    x, q = _dev(cfg["xyz"]), _dev(cfg["q"])
    F = torch.empty_like(x)
    for _ in range(3):
        e.forces_device(x, q, F)
    # new coordinates in the same buffer
    rng = np.random.default_rng(8)
    xyz2 = cfg["xyz"] + rng.normal(scale=0.05, size=cfg["xyz"].shape)
    xyz2[:, 2] = np.clip(xyz2[:, 2], 0.6, 9.4)
    x.copy_(_dev(xyz2))
    e.forces_device(x, q, F)
    assert np.array_equal(F.cpu().numpy(), e.forces(xyz2, cfg["q"]))
    # a new k-set
    e.sample_kset(123, cfg["P"])
    for _ in range(3):
        e.forces_device(x, q, F)
    assert np.array_equal(F.cpu().numpy(), e.forces(xyz2, cfg["q"]))
    # another output buffer
    F2 = torch.empty_like(x)
    for _ in range(3):
        e.forces_device(x, q, F2)
    assert np.array_equal(F2.cpu().numpy(), F.cpu().numpy())


def test_replay_overflow_and_status():
    import torch

    rng = np.random.default_rng(5)
    N, Lb = 1500, (200.0, 200.0, 10.0)
    spread = np.stack([Lb[0] * rng.random(N), Lb[1] * rng.random(N), 0.5 + 9 * rng.random(N)], 1)
    packed = np.stack([50 + 20 * rng.random(N), 80 + 20 * rng.random(N), 0.5 + 9 * rng.random(N)], 1)
    qh = np.where(np.arange(N) < N // 2, 1.0, -1.0)
    cfg = dict(L=Lb, alpha=0.1, r_cutoff=10.0, gamma_down=0.5, gamma_up=-0.4, accuracy=1e-6, N_t=30, P=40,
               walls=[])
    e = W.engine_for(cfg, "fp64")
    x, q = _dev(spread), _dev(qh)
    F = torch.empty_like(x)
    for _ in range(3):
        e.forces_device(x, q, F)
    x.copy_(_dev(packed))                            # 20x the pairs: the replay overflows
    e.forces_device(x, q, F)
    fresh = W.engine_for(cfg, "fp64")
    assert np.array_equal(F.cpu().numpy(), fresh.forces(packed, qh))
    for _ in range(2):
        e.forces_device(x, q, F)
    assert np.array_equal(F.cpu().numpy(), fresh.forces(packed, qh))
    bad = packed.copy()
    bad[7, 0] = np.nan
    x.copy_(_dev(bad))
    with pytest.raises(L.QemError):
        e.forces_device(x, q, F)
    x.copy_(_dev(packed))
    e.forces_device(x, q, F)
    assert np.array_equal(F.cpu().numpy(), fresh.forces(packed, qh))


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_pinned_host_buffers_replay(prec):
    import torch

    cfg = W.config3(N=4000)
    e = W.engine_for(cfg, prec)
    ref = e.forces(cfg["xyz"], cfg["q"])
    xh = torch.tensor(cfg["xyz"], dtype=torch.float64).pin_memory()
    qh = torch.tensor(cfg["q"], dtype=torch.float64).pin_memory()
    Fh = torch.empty_like(xh).pin_memory()
    for _ in range(4):                              # ordinary, record + replay, replay, replay
        Fh.fill_(float("nan"))
        e.forces(xh.numpy(), qh.numpy(), out=Fh.numpy())
        assert np.array_equal(Fh.numpy(), ref)
    rng = np.random.default_rng(9)
    xyz2 = cfg["xyz"] + rng.normal(scale=0.05, size=cfg["xyz"].shape)
    xyz2[:, 2] = np.clip(xyz2[:, 2], 0.6, 9.4)
    xh.copy_(torch.tensor(xyz2))                    # new coordinates in the same page-locked buffer
    e.forces(xh.numpy(), qh.numpy(), out=Fh.numpy())
    got = Fh.numpy().copy()
    assert np.array_equal(got, e.forces(xyz2, cfg["q"]))
    # the device-memory graph of the same handle and the host one agree
    x, q = _dev(xyz2), _dev(cfg["q"])
    F = torch.empty_like(x)
    for _ in range(3):
        e.forces_device(x, q, F)
    assert np.array_equal(F.cpu().numpy(), got)
