"""Seeded synthetic slab systems with the shapes of the benchmark configurations.

Each generator returns a dict with coordinates (N x 3), charges (N), box L,
and the QEM parameters.  Charges are exactly neutral.  Seeds are fixed
(20261203 + config index) so every run sees the same systems.
"""
from __future__ import annotations

import numpy as np

SEED0 = 20261203


def _slab(rng, N, Lx, Ly, zlo, zhi):
    return np.stack([rng.random(N) * Lx, rng.random(N) * Ly, zlo + rng.random(N) * (zhi - zlo)], axis=1)


def _hard_core_slab(rng, N, Lx, Ly, zlo, zhi, dmin):
    """Uniform slab positions, each redrawn until it is at least dmin (3-D,
    minimum image in x and y) from every earlier particle."""
    xyz = _slab(rng, N, Lx, Ly, zlo, zhi)
    cell = max(dmin, 1e-9)
    grid = {}
    for i in range(N):
        while True:
            p = xyz[i]
            cx, cy, cz = int(p[0] // cell), int(p[1] // cell), int(p[2] // cell)
            ok = True
            for dx in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for dz in (-1, 0, 1):
                        for j in grid.get(((cx + dx) % max(1, int(Lx // cell)), (cy + dy) % max(1, int(Ly // cell)),
                                           cz + dz), ()):
                            d = xyz[j] - p
                            d[0] -= Lx * np.rint(d[0] / Lx)
                            d[1] -= Ly * np.rint(d[1] / Ly)
                            if d @ d < dmin * dmin:
                                ok = False
            if ok:
                break
            xyz[i] = _slab(rng, 1, Lx, Ly, zlo, zhi)[0]
        key = (cx % max(1, int(Lx // cell)), cy % max(1, int(Ly // cell)), cz)
        grid.setdefault(key, []).append(i)
    return xyz


def _pm_charges(N):
    q = np.ones(N)
    q[N // 2:] = -1.0
    if N % 2:
        q[-1] = 0.0
    return q


def config1(seed=None):
    """N=100 (50 +1, 50 -1), Lx=Ly=100, Lz=10, gamma_up=0.95, gamma_down=-0.95, alpha=0.1, r_c=10,
    N_t=30, P=100, LJ walls at z=0 (+1) and z=10 (-1) with eps=1, sigma=1, cutoff=1."""
    rng = np.random.default_rng(SEED0 + 1 if seed is None else seed)
    N = 100
    return dict(name="config1_N100_slab", N=N, L=(100.0, 100.0, 10.0), xyz=_slab(rng, N, 100.0, 100.0, 0.5, 9.5),
                q=_pm_charges(N), alpha=0.1, r_cutoff=10.0, gamma_up=0.95, gamma_down=-0.95, N_t=30,
                accuracy=1e-6, P=100,
                walls=[dict(cutoff=1.0, sigma=1.0, eps=1.0, sub_pos=0.0, direction=+1),
                       dict(cutoff=1.0, sigma=1.0, eps=1.0, sub_pos=10.0, direction=-1)])


def config2(seed=None, N=100_000):
    """N=1e5 (+-1, neutral), Lx=Ly=1000, Lz=10, z in [0.5, 9.5], gamma_up=gamma_down=0.95,
    alpha=0.1, r_c=10, P=500 (about 31 neighbours within r_c)."""
    rng = np.random.default_rng(SEED0 + 2 if seed is None else seed)
    L = 1000.0 * np.sqrt(N / 100_000)
    return dict(name=f"config2_N{N}_slab", N=N, L=(L, L, 10.0), xyz=_slab(rng, N, L, L, 0.5, 9.5),
                q=_pm_charges(N), alpha=0.1, r_cutoff=10.0, gamma_up=0.95, gamma_down=0.95, N_t=30,
                accuracy=1e-6, P=500, walls=[])


def config3(seed=None, N=20_000):
    """N=2e4, |q| ~ U[0.5, 1.5] with random sign, re-neutralised; Lx=Ly=450, Lz=10,
    gamma_up=0.8, gamma_down=-0.6."""
    rng = np.random.default_rng(SEED0 + 3 if seed is None else seed)
    L = 450.0 * np.sqrt(N / 20_000)
    q = rng.uniform(0.5, 1.5, N) * rng.choice([-1.0, 1.0], N)
    q[-1] -= q.sum()
    return dict(name=f"config3_N{N}_slab", N=N, L=(L, L, 10.0), xyz=_slab(rng, N, L, L, 0.5, 9.5), q=q,
                alpha=0.1, r_cutoff=10.0, gamma_up=0.8, gamma_down=-0.6, N_t=30, accuracy=1e-6, P=500, walls=[])


def config4(seed=None, n_systems=256):
    """256 independent slabs, N ~ U[200, 5000], Lz ~ U[5, 20], Lx=Ly from density 0.01,
    gamma pairs ~ U(-0.95, 0.95)^2, alpha=0.1, r_c=10, P=200.  Positions are uniform
    with a hard core of 1.0 (no two particles closer), so that the bare +-1 charges
    (no Lennard-Jones core between particles) do not collapse onto each other within
    a 1000-step, dt = 1e-3 velocity-Verlet run."""
    rng = np.random.default_rng(SEED0 + 4 if seed is None else seed)
    out = []
    for s in range(n_systems):
        N = int(rng.integers(200, 5001))
        Lz = float(rng.uniform(5, 20))
        L = float(np.sqrt(N / 0.01))
        gu, gd = rng.uniform(-0.95, 0.95, 2)
        out.append(dict(name=f"config4_sys{s}", N=N, L=(L, L, Lz), xyz=_hard_core_slab(rng, N, L, L, 0.5, Lz - 0.5, 1.0),
                        q=_pm_charges(N), alpha=0.1, r_cutoff=10.0, gamma_up=float(gu), gamma_down=float(gd),
                        N_t=30, accuracy=1e-6, P=200, walls=[]))
    return out


def config5(seed=None, N=1_000_000):
    """N=1e6 (+-1), Lx=Ly=3162, Lz=10, gamma_up=gamma_down=0.99, alpha=0.1, r_c=10, P=2000."""
    rng = np.random.default_rng(SEED0 + 5 if seed is None else seed)
    L = 3162.0 * np.sqrt(N / 1_000_000)
    return dict(name=f"config5_N{N}_slab", N=N, L=(L, L, 10.0), xyz=_slab(rng, N, L, L, 0.5, 9.5),
                q=_pm_charges(N), alpha=0.1, r_cutoff=10.0, gamma_up=0.99, gamma_down=0.99, N_t=30,
                accuracy=1e-6, P=2000, walls=[])


def engine_for(cfg, precision="fp64", mode_flags=0, seed=7, device=0):
    """A libqem Engine configured for cfg, with a seeded k-set of cfg['P'] vectors."""
    from . import _lib as L
    from .api import Engine, Substrate_LJ

    walls = [Substrate_LJ(**w) for w in cfg.get("walls", [])]
    e = Engine(L_box=cfg["L"], alpha=cfg["alpha"], r_cutoff=cfg["r_cutoff"], gamma_1=cfg["gamma_down"],
               gamma_2=cfg["gamma_up"], accuracy=cfg["accuracy"], N_t=cfg["N_t"], rbe_p=cfg["P"], walls=walls,
               mode_flags=mode_flags, precision={"fp64": L.QEM_FP64, "fp32": L.QEM_FP32_FIX}[precision],
               device=device)
    e.sample_kset(seed, cfg["P"])
    return e


def rel_err(F, Fref):
    """(||F - Fref||_2 / ||Fref||_2, max_i |F_i - Fref_i| / rms_i |Fref_i|) over all particles."""
    d = np.asarray(F) - np.asarray(Fref)
    nref = np.linalg.norm(Fref)
    rms = nref / np.sqrt(max(len(Fref), 1))
    return float(np.linalg.norm(d) / nref), float(np.max(np.linalg.norm(d, axis=1)) / rms)


def main(argv=None):
    """Run a few force evaluations of a workload on cuda:0 (profiling target).

    python -m qem4molly_b200.workloads --config 2 --evals 3 --precision fp32
    """
    import argparse

    import torch

    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--config", type=int, default=2, choices=(1, 2, 3, 4, 5),
                    help="4: the 256-slab batch in fused phases (FP32+fix, a fresh k batch per evaluation)")
    ap.add_argument("--evals", type=int, default=3)
    ap.add_argument("--precision", default="fp32", choices=("fp32", "fp64"))
    ap.add_argument("--N", type=int, default=None, help="particle count (configs 2, 3, 5)")
    ap.add_argument("--ties", type=float, default=0.0,
                    help="round z to multiples of this spacing and evaluate with QEM_EQUAL_Z_TIES")
    ap.add_argument("--norm", action="store_true",
                    help="gamma_1 = gamma_2 = e with Lz = 2 (regularised quadrature, python mode, FP64)")
    ap.add_argument("--backward", action="store_true",
                    help="time qem_backward (FP64) for loss = E + sum_i w_i . F_i, w ~ N(0, 1), instead")
    ap.add_argument("--tiling", type=int, nargs=3, default=(4, 0, 64), metavar=("KS", "ORDER", "CHUNK"),
                    help="config 4: fused tiling (k-slices per system, work-list order, chunk length)")
    a = ap.parse_args(argv)
    from . import _lib as L

    if a.config == 4:
        from .api import Batch

        cfgs = config4()
        engines = [engine_for(c, "fp32", mode_flags=L.QEM_RESAMPLE_KSET, seed=100 + i) for i, c in enumerate(cfgs)]
        dev = torch.device("cuda", 0)
        x = torch.tensor(np.concatenate([c["xyz"] for c in cfgs]), device=dev)
        q = torch.tensor(np.concatenate([c["q"] for c in cfgs]), device=dev)
        F = torch.empty_like(x)
        b = Batch(engines, [c["N"] for c in cfgs])
        b.set_mode(L.QEM_BATCH_FUSED, *a.tiling)
        b.forces(x, q, F)  # synchronous sizing pass
        for _ in range(a.evals):
            b.forces(x, q, F)
        b.check()
        print(f"config 4: {len(cfgs)} slabs, {x.shape[0]} particles, {a.evals} fused evaluations, {b.mode()}")
        return

    make = {1: config1, 2: config2, 3: config3, 5: config5}[a.config]
    cfg = make(N=a.N) if (a.N and a.config != 1) else make()
    if a.ties > 0:
        cfg["xyz"][:, 2] = np.round(cfg["xyz"][:, 2] / a.ties) * a.ties
    if a.norm:
        from .api import Engine

        cfg["L"] = (cfg["L"][0], cfg["L"][1], 2.0)
        cfg["xyz"][:, 2] = 0.2 + 1.6 * (cfg["xyz"][:, 2] - cfg["xyz"][:, 2].min()) / np.ptp(cfg["xyz"][:, 2])
        e = Engine(L_box=cfg["L"], alpha=cfg["alpha"], r_cutoff=cfg["r_cutoff"], gamma_1=np.e, gamma_2=np.e,
                   accuracy=cfg["accuracy"], N_t=cfg["N_t"], rbe_p=cfg["P"], mode_flags=L.QEM_PYTHON_MODE,
                   precision=L.QEM_FP64, pv_eps=0.05)
        e.sample_kset(7, cfg["P"])
        a.precision = "fp64 (gamma_1 gamma_2 = e^2, Lz = 2, regularised)"
    else:
        e = engine_for(cfg, a.precision, mode_flags=L.QEM_EQUAL_Z_TIES if a.ties > 0 else 0)
    dev = torch.device("cuda", 0)
    x = torch.tensor(cfg["xyz"], dtype=torch.float64, device=dev)
    q = torch.tensor(cfg["q"], dtype=torch.float64, device=dev)
    F = torch.empty_like(x)
    if a.backward:
        w = torch.tensor(np.random.default_rng(SEED0 + 6).normal(size=cfg["xyz"].shape), device=dev)
        gx, gq = torch.empty_like(x), torch.empty_like(q)
        for _ in range(a.evals):
            e.backward_device(x, q, w, 1.0, gx, gq)
        torch.cuda.synchronize()
        print(f"config {a.config}: N={len(cfg['q'])}, {a.evals} backward passes, |dL/dr|_max={gx.abs().max().item():.6e}")
        return
    for _ in range(3):
        e.forces_device(x, q, F)
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record()
    for _ in range(a.evals):
        e.forces_device(x, q, F)
    t1.record()
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1) / max(a.evals, 1)
    print(f"config {a.config}: N={len(cfg['q'])}, {a.evals} {a.precision} evaluations "
          f"{'with equal-z ties ' if a.ties > 0 else ''}(back to back, {ms:.3f} ms each), "
          f"|F|_max={F.abs().max().item():.6e}")


if __name__ == "__main__":
    main()
