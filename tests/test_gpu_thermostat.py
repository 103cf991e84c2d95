"""Andersen thermostat of the batch MD (qem_batch_set_thermostat; Molly
AndersenThermostat(temp, coupling_const) as in test/QEM_test.jl:53-56, python_lib
Andersen.py:8-22): one thermostatted step against a host restatement of the
counter-based draws (collision choices bit for bit, new velocities to rounding),
the collision rate, the velocity distribution at p = 1, the step counter, and
thermostat-off runs identical to plain MD."""
import numpy as np
import pytest

from qem4molly_b200 import workloads as W
from qem4molly_b200.api import Batch

pytestmark = pytest.mark.gpu

C1, C2 = np.uint64(0xBF58476D1CE4E5B9), np.uint64(0x94D049BB133111EB)
G = np.uint64(0x9E3779B97F4A7C15)


def _mix(z):
    z = (z ^ (z >> np.uint64(30))) * C1
    z = (z ^ (z >> np.uint64(27))) * C2
    return z ^ (z >> np.uint64(31))


def _unit(seed, step, i, k):
    """u in (0, 1] of draw k of particle i at a step (the library's counter-based generator)."""
    with np.errstate(over="ignore"):
        s = np.uint64(seed) + G * np.uint64(step + 1)
        r = _mix(_mix(_mix(np.full(i.shape, s, dtype=np.uint64)) + G * (i + np.uint64(1))) + G * np.uint64(k + 1))
    return ((r >> np.uint64(11)).astype(np.float64) + 1.0) * 2.0 ** -53


def _setup(n_sys=4):
    import torch

    cfgs = W.config4(n_systems=n_sys)
    engines = [W.engine_for(c, "fp64", seed=100 + i) for i, c in enumerate(cfgs)]
    N = [c["N"] for c in cfgs]
    x0 = np.concatenate([c["xyz"] for c in cfgs])
    q = torch.tensor(np.concatenate([c["q"] for c in cfgs]), device="cuda")
    v0 = np.random.default_rng(5).normal(scale=0.3, size=x0.shape)
    return engines, N, x0, v0, q


def _run(b, x0, v0, q, steps, dt):
    import torch

    x = torch.tensor(x0, device="cuda")
    v = torch.tensor(v0, device="cuda")
    F = torch.empty_like(x)
    b.md(steps, dt, x, v, q, F)
    return x.cpu().numpy(), v.cpu().numpy()


def test_one_step_matches_host_draws():
    engines, N, x0, v0, q = _setup()
    b = Batch(engines, N)
    dt, kT, nu, seed = 1e-3, 2.0, 50.0, 123
    x_plain, v_plain = _run(b, x0, v0, q, 1, dt)
    b.set_thermostat(kT, nu, seed)
    x_t, v_t = _run(b, x0, v0, q, 1, dt)
    assert b.thermostat_step() == 1
    assert np.array_equal(x_t, x_plain)  # the thermostat acts after the velocity update only
    n = x0.shape[0]
    i = np.arange(n, dtype=np.uint64)
    p = nu * dt
    sel = _unit(seed, 0, i, 0) <= p
    assert np.array_equal(v_t[~sel], v_plain[~sel])
    u1, u2, u3, u4 = (_unit(seed, 0, i, k) for k in (1, 2, 3, 4))
    r1, r2 = np.sqrt(kT) * np.sqrt(-2 * np.log(u1)), np.sqrt(kT) * np.sqrt(-2 * np.log(u3))
    vn = np.stack([r1 * np.cos(2 * np.pi * u2), r1 * np.sin(2 * np.pi * u2), r2 * np.cos(2 * np.pi * u4)], 1)
    np.testing.assert_allclose(v_t[sel], vn[sel], rtol=1e-12, atol=1e-13)
    k = int(sel.sum())
    assert abs(k - p * n) <= 5 * np.sqrt(n * p * (1 - p)), (k, p * n)
    assert not np.array_equal(v_t[sel], v_plain[sel])


def test_full_resampling_distribution_and_counter():
    engines, N, x0, v0, q = _setup()
    b = Batch(engines, N)
    dt, kT = 1e-3, 0.7
    b.set_thermostat(kT, 1.0 / dt, 9)  # p = 1: every velocity is redrawn every step
    _, v1 = _run(b, x0, v0, q, 1, dt)
    n = v1.size
    assert abs(v1.mean()) <= 5 * np.sqrt(kT / n)
    assert abs(v1.var() / kT - 1) <= 5 * np.sqrt(2.0 / n)
    assert b.thermostat_step() == 1
    _, v2 = _run(b, x0, v0, q, 2, dt)  # the counter continues: new draws
    assert b.thermostat_step() == 3
    assert not np.allclose(v2, v1)
    b.set_thermostat(kT, 1.0 / dt, 9)  # reset: the first step's draws again
    _, v1b = _run(b, x0, v0, q, 1, dt)
    assert np.array_equal(v1b, v1)


def test_thermostat_off_is_plain_md():
    engines, N, x0, v0, q = _setup(3)
    b = Batch(engines, N)
    xa, va = _run(b, x0, v0, q, 3, 1e-3)
    b.set_thermostat(1.0, 0.0, 1)  # nu = 0: off
    xb, vb = _run(b, x0, v0, q, 3, 1e-3)
    assert np.array_equal(xa, xb) and np.array_equal(va, vb)
    assert b.thermostat_step() == 0
