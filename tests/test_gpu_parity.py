"""GPU parity: libqem.so (through its C-ABI) against the FP64 CPU oracle.

Tolerances (stated per test):
  * integer work (cells, pair list, z order): bit-exact;
  * FP64 path: relative L2 force error <= 1e-11 for the short range and
    <= 1e-9 for the long range (the oracle restates the reference's
    "total minus running sum" suffix sums, Force_long.jl:97-98, whose own
    rounding is ~eps * e^{k L_z}); energies <= 1e-11 relative;
  * FP32+fix path: relative L2 force error <= 1e-5 (the metric's bound).
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from qem4molly_b200 import _lib as L
from qem4molly_b200 import workloads as W
from qem4molly_b200.api import Engine, Substrate_LJ

pytestmark = pytest.mark.gpu


def slab(N, Lb, seed, zlo=0.5, zhi=None, charges="pm"):
    rng = np.random.default_rng(seed)
    Lx, Ly, Lz = Lb
    zhi = Lz - 0.5 if zhi is None else zhi
    xyz = np.stack([rng.random(N) * Lx, rng.random(N) * Ly, zlo + rng.random(N) * (zhi - zlo)], 1)
    if charges == "pm":
        q = np.where(np.arange(N) < N // 2, 1.0, -1.0)
    else:
        q = rng.uniform(0.5, 1.5, N) * rng.choice([-1.0, 1.0], N)
        q[-1] -= q.sum()
    return xyz, q


def oparams(Lb, alpha, rc, gd, gu, flags=0, N_t=30, acc=1e-6):
    return O.params(Lb, alpha, rc, gd, gu, accuracy=acc, N_t=N_t,
                    cutoff_mode=1 if flags & L.QEM_CUTOFF_PYTHON else 0,
                    dir_mode=1 if flags & L.QEM_DIR_MINIMAGE else 0,
                    pair_mode=1 if flags & L.QEM_PAIR_PHYSICAL else 0)


def kset_of(e):
    k3, sK = e.get_kset()
    return k3, sK


# ---------------------------------------------------------------- integer work
@pytest.mark.parametrize("Lb,rc", [((100.0, 100.0, 10.0), 10.0), ((25.0, 25.0, 10.0), 10.0),
                                   ((33.0, 47.0, 5.0), 10.0), ((200.0, 90.0, 10.0), 7.5),
                                   ((1000.0, 1000.0, 10.0), 10.0)])
def test_pair_list_bitexact(Lb, rc):
    """Pair set equal to the brute-force oracle's: dense boxes (one warp per owner cell),
    a box with 2 cells along an axis (full stencil) and a sparse box (one thread per owner)."""
    xyz, _ = slab(3000, Lb, 11)
    xyz[:7, :2] -= np.array([Lb[0], 0.0])  # some coordinates outside [0, L): wrapped by the binning
    e = Engine(L_box=Lb, alpha=0.1, r_cutoff=rc, rbe_p=0)
    got = e.pair_list(xyz)
    ref = O.pairs(oparams(Lb, 0.1, rc, 0, 0), xyz, method="brute")
    g = np.sort(got[:, 0].astype(np.int64) * 10**6 + got[:, 1])
    r = np.sort(ref[:, 0].astype(np.int64) * 10**6 + ref[:, 1])
    assert np.array_equal(g, r)
    assert np.all(got[:, 0] < got[:, 1])


def test_cell_index_matches_definition():
    Lb = (100.0, 80.0, 10.0)
    xyz, _ = slab(5000, Lb, 12)
    e = Engine(L_box=Lb, alpha=0.1, r_cutoff=10.0, rbe_p=0)
    cell, start, (ncx, ncy) = e.cell_index(xyz)
    assert (ncx, ncy) == (10, 8)
    xw = xyz[:, 0] - Lb[0] * np.floor(xyz[:, 0] * (1 / Lb[0]))
    yw = xyz[:, 1] - Lb[1] * np.floor(xyz[:, 1] * (1 / Lb[1]))
    cx = np.clip((xw * (ncx / Lb[0])).astype(int), 0, ncx - 1)
    cy = np.clip((yw * (ncy / Lb[1])).astype(int), 0, ncy - 1)
    assert np.array_equal(cell, cx * ncy + cy)
    assert np.array_equal(np.diff(start), np.bincount(cell, minlength=ncx * ncy))


@pytest.mark.parametrize("N,kind", [(1, "uniform"), (1000, "uniform"), (5000, "ties"), (70_000, "ties"),
                                    (100_000, "uniform"), (30_000, "outside")])
def test_z_order_is_sortperm(N, kind):
    """QEM_long.jl:39-40 sortperm: stable ascending, ties in index order.  Up
    to 2048 particles one tile pass; above, the z-bucket passes (uniform z,
    ties of about 135 particles per z value, particles outside [0, L_z]),
    or the tile and merge passes behind them when a bucket overflows (ties of
    about 1900 particles per z value at N = 7e4)."""
    xyz, _ = slab(N, (300.0, 300.0, 10.0), 13)
    if kind == "ties":
        xyz[:, 2] = np.round(xyz[:, 2] * 4) / 4
    if kind == "outside":
        xyz[:50, 2] = -3.0
        xyz[50:100, 2] = 14.0
    e = Engine(L_box=(300.0, 300.0, 10.0), alpha=0.1, r_cutoff=10.0, rbe_p=0)
    assert np.array_equal(e.z_order(xyz), np.argsort(xyz[:, 2], kind="stable"))
    assert np.array_equal(e.z_order(xyz), O.sortperm_z(xyz))


# ---------------------------------------------------------------- FP64 parity
MODES = [0, L.QEM_PYTHON_MODE, L.QEM_PAIR_PHYSICAL, L.QEM_DIR_MINIMAGE]


@pytest.mark.parametrize("flags", MODES)
def test_short_fp64_vs_oracle(flags):
    Lb = (60.0, 60.0, 10.0)
    xyz, q = slab(300, Lb, 21, charges="uniform")
    gd, gu = -0.6, 0.8
    e = Engine(L_box=Lb, alpha=0.1, r_cutoff=10.0, gamma_1=gd, gamma_2=gu, rbe_p=0, mode_flags=flags)
    F = e.forces(xyz, q, terms=L.QEM_TERM_SHORT)
    p = oparams(Lb, 0.1, 10.0, gd, gu, flags)
    Fref = O.short_forces(p, xyz, q)
    assert W.rel_err(F, Fref)[0] <= 1e-11


def test_long_fp64_vs_oracle():
    Lb = (40.0, 40.0, 10.0)
    xyz, q = slab(500, Lb, 22, charges="uniform")
    e = Engine(L_box=Lb, alpha=0.1, r_cutoff=10.0, gamma_1=0.95, gamma_2=0.9, rbe_p=60)
    e.sample_kset(5, 60)
    F = e.forces(xyz, q, terms=L.QEM_TERM_LONG)
    k3, sK = kset_of(e)
    Fref = O.F_long(oparams(Lb, 0.1, 10.0, 0.95, 0.9), xyz, q, k3, sK)
    assert W.rel_err(F, Fref)[0] <= 1e-9


def test_energy_fp64_vs_oracle():
    Lb = (50.0, 50.0, 8.0)
    xyz, q = slab(250, Lb, 23, charges="uniform")
    for flags in (0, L.QEM_PYTHON_MODE):
        e = Engine(L_box=Lb, alpha=0.1, r_cutoff=10.0, gamma_1=-0.7, gamma_2=0.9, rbe_p=40, mode_flags=flags)
        e.sample_kset(3, 40)
        k3, sK = kset_of(e)
        p = oparams(Lb, 0.1, 10.0, -0.7, 0.9, flags)
        Es = e.energy(xyz, q, terms=L.QEM_TERM_SHORT)
        El = e.energy(xyz, q, terms=L.QEM_TERM_LONG)
        assert np.isclose(Es, O.energy_short(p, xyz, q), rtol=1e-11)
        assert np.isclose(El, O.energy_long(p, xyz, q, k3, sK), rtol=1e-10)


def test_walls_vs_oracle():
    cfg = W.config1()
    e = W.engine_for(cfg)
    F = e.forces(cfg["xyz"], cfg["q"], terms=L.QEM_TERM_LJ)
    Fref, bad = O.lj_two_walls(cfg["xyz"], cfg["walls"])
    # 2 s^12 - s^6 cancels near the LJ minimum: compare against the largest wall force
    assert bad == 0 and np.allclose(F, Fref, rtol=1e-13, atol=1e-14 * np.abs(Fref).max())


def test_config1_total_fp64():
    """Config 1 (N=100): short + self + long + walls against the oracle."""
    cfg = W.config1()
    e = W.engine_for(cfg)
    F, E = e.forces(cfg["xyz"], cfg["q"], energy=True)
    k3, sK = kset_of(e)
    p = oparams(cfg["L"], cfg["alpha"], cfg["r_cutoff"], cfg["gamma_down"], cfg["gamma_up"])
    Fref = O.short_forces(p, cfg["xyz"], cfg["q"]) + O.F_long(p, cfg["xyz"], cfg["q"], k3, sK)
    Fref += O.lj_two_walls(cfg["xyz"], cfg["walls"])[0]
    assert W.rel_err(F, Fref)[0] <= 1e-10
    Eref = O.energy_short(p, cfg["xyz"], cfg["q"]) + O.energy_long(p, cfg["xyz"], cfg["q"], k3, sK)
    assert np.isclose(E, Eref, rtol=1e-10)


# ---------------------------------------------------------------- FP32+fix path
@pytest.mark.parametrize("cfgname", ["config1", "config2s", "config3s", "gamma099"])
def test_fp32_fix_force_error(cfgname):
    if cfgname == "config1":
        cfg = W.config1()
    elif cfgname == "config2s":
        cfg = W.config2(N=4000)
    elif cfgname == "config3s":
        cfg = W.config3(N=4000)
    else:
        cfg = W.config2(N=4000)
        cfg["gamma_up"] = cfg["gamma_down"] = 0.99
    e64 = W.engine_for(cfg, "fp64")
    e32 = W.engine_for(cfg, "fp32")
    F64, E64 = e64.forces(cfg["xyz"], cfg["q"], energy=True)
    F32, E32 = e32.forces(cfg["xyz"], cfg["q"], energy=True)
    k3, sK = kset_of(e64)
    p = oparams(cfg["L"], cfg["alpha"], cfg["r_cutoff"], cfg["gamma_down"], cfg["gamma_up"])
    Fref = O.short_forces(p, cfg["xyz"], cfg["q"]) + O.F_long(p, cfg["xyz"], cfg["q"], k3, sK)
    if cfg["walls"]:
        Fref += O.lj_two_walls(cfg["xyz"], cfg["walls"])[0]
    assert W.rel_err(F64, Fref)[0] <= 1e-9
    assert W.rel_err(F32, Fref)[0] <= 1e-5
    assert abs(E32 - E64) <= 1e-5 * abs(E64)


# ---------------------------------------------------------------- edge cases
def test_empty_and_single():
    e = Engine(L_box=(50.0, 50.0, 10.0), alpha=0.1, r_cutoff=10.0, gamma_1=0.5, gamma_2=0.5, rbe_p=10)
    F, E = e.forces(np.zeros((0, 3)), np.zeros(0), energy=True)
    assert F.shape == (0, 3) and E == 0.0
    xyz = np.array([[10.0, 10.0, 3.0]])
    F, E = e.forces(xyz, np.array([1.0]), energy=True)
    p = oparams((50.0, 50.0, 10.0), 0.1, 10.0, 0.5, 0.5)
    k3, sK = kset_of(e)
    Fref = O.short_forces(p, xyz, np.array([1.0])) + O.F_long(p, xyz, np.array([1.0]), k3, sK)
    assert np.allclose(F, Fref, rtol=1e-10, atol=1e-14)


def test_rho_zero_pair_and_nonneutral():
    """A pair on the same vertical line (rho = 0: Force_short.jl:46 skips x/y) and net charge."""
    Lb = (30.0, 30.0, 10.0)
    xyz = np.array([[5.0, 5.0, 2.0], [5.0, 5.0, 6.0], [9.0, 7.0, 4.0]])
    q = np.array([1.0, 1.0, -0.5])
    e = Engine(L_box=Lb, alpha=0.1, r_cutoff=8.0, gamma_1=0.3, gamma_2=-0.4, rbe_p=20)
    e.sample_kset(1, 20)
    F = e.forces(xyz, q)
    k3, sK = kset_of(e)
    p = oparams(Lb, 0.1, 8.0, 0.3, -0.4)
    Fref = O.short_forces(p, xyz, q) + O.F_long(p, xyz, q, k3, sK)
    assert W.rel_err(F, Fref)[0] <= 1e-10


def test_errors_are_status_codes():
    e = Engine(L_box=(50.0, 50.0, 10.0), alpha=0.1, r_cutoff=10.0, rbe_p=10,
               walls=[Substrate_LJ(cutoff=1.0, sigma=1.0, eps=1.0, sub_pos=0.0, direction=+1)])
    xyz, q = slab(50, (50.0, 50.0, 10.0), 31)
    bad = xyz.copy()
    bad[3, 1] = np.nan
    with pytest.raises(L.QemError) as ei:
        e.forces(bad, q)
    assert ei.value.status == 3
    out = xyz.copy()
    out[5, 2] = -0.2  # below the z = 0 wall: Substrate_LJ.jl:37
    with pytest.raises(L.QemError) as ei:
        e.forces(out, q)
    assert ei.value.status == 2
    F = e.forces(xyz, q)  # the handle stays usable
    assert np.all(np.isfinite(F))
    with pytest.raises(ValueError):
        e.forces(xyz, q[:-1])


def test_stale_neighbor_list_semantics():
    """QEM_short.jl:32-36: the list is rebuilt on calls 1, 1 + iter_period, ...; in between,
    pairs that left r_c give zero (Force_short.jl:36-39) and new pairs are missed."""
    Lb = (60.0, 60.0, 10.0)
    xyz0, q = slab(200, Lb, 41)
    e = Engine(L_box=Lb, alpha=0.1, r_cutoff=8.0, gamma_1=0.5, gamma_2=0.5, rbe_p=0, iter_period=3,
               mode_flags=L.QEM_STALE_NEIGHBORS)
    p = oparams(Lb, 0.1, 8.0, 0.5, 0.5)
    rng = np.random.default_rng(5)
    pl = None
    xyz = xyz0.copy()
    for call in range(5):
        if call % 3 == 0:
            pl = O.pairs(p, xyz)
        F = e.forces(xyz, q, terms=L.QEM_TERM_SHORT)
        assert W.rel_err(F, O.short_forces(p, xyz, q, pl))[0] <= 1e-11
        xyz[:, :2] = (xyz[:, :2] + rng.normal(0, 1.5, (len(xyz), 2))) % 60.0


def test_bitwise_repeatable():
    cfg = W.config2(N=3000)
    for prec in ("fp64", "fp32"):
        e = W.engine_for(cfg, prec)
        a = e.forces(cfg["xyz"], cfg["q"], energy=True)
        b = e.forces(cfg["xyz"], cfg["q"], energy=True)
        assert np.array_equal(a[0], b[0]) and a[1] == b[1]


def test_kset_sampler_distribution():
    """Separable sampling of exp(-k^2 / 4 alpha) on the lattice (K_set_generator.jl:30-41)."""
    Lb = (30.0, 30.0, 10.0)
    e = Engine(L_box=Lb, alpha=0.1, r_cutoff=5.0, rbe_p=200_000)
    e.sample_kset(123, 200_000)
    k3, sK = kset_of(e)
    K, P, sum_K = O.kset_generator(30.0, 30.0, 0.1, 1e-6)
    assert np.isclose(sK, sum_K, rtol=1e-12)
    m = np.rint(k3[:, :2] * 30.0 / (2 * np.pi)).astype(int)
    assert not np.any((m[:, 0] == 0) & (m[:, 1] == 0))
    mref = np.rint(K[:, :2] * 30.0 / (2 * np.pi)).astype(int)
    key = lambda a: a[:, 0] * 1000 + a[:, 1]
    pref = dict(zip(key(mref), P.astype(np.float64)))
    vals, cnt = np.unique(key(m), return_counts=True)
    expected = np.array([pref[v] for v in vals]) * len(m)
    sel = expected > 50
    chi2 = np.sum((cnt[sel] - expected[sel]) ** 2 / expected[sel])
    assert chi2 / sel.sum() < 2.0


# ---------------------------------------------------------------- device path, torch
def test_device_path_and_autograd():
    import torch

    from qem4molly_b200.torch_fn import QEMEnergyForces

    cfg = W.config2(N=2000)
    e = W.engine_for(cfg, "fp64")
    Fh, Eh = e.forces(cfg["xyz"], cfg["q"], terms=L.QEM_TERM_SHORT | L.QEM_TERM_LONG, energy=True)
    x = torch.tensor(cfg["xyz"], device="cuda", dtype=torch.float64, requires_grad=True)
    q = torch.tensor(cfg["q"], device="cuda", dtype=torch.float64)
    E, F = QEMEnergyForces.apply(x, q, e)
    assert np.array_equal(F.detach().cpu().numpy(), Fh) and float(E.detach()) == Eh
    E.backward()
    gx, _, _ = e.backward(cfg["xyz"], cfg["q"], None, 1.0, terms=L.QEM_TERM_SHORT | L.QEM_TERM_LONG)
    assert np.array_equal(x.grad.cpu().numpy(), gx)


# ---------------------------------------------------------------- full size properties
def test_config2_full_size_properties():
    """N = 1e5 (the benchmark system): FP32+fix vs FP64 within 1e-5, repeatable, and
    invariant under an in-plane translation (minimum-image mode) to FP64 rounding."""
    cfg = W.config2()
    e64 = W.engine_for(cfg, "fp64")
    e32 = W.engine_for(cfg, "fp32")
    F64, E64 = e64.forces(cfg["xyz"], cfg["q"], energy=True)
    F32, E32 = e32.forces(cfg["xyz"], cfg["q"], energy=True)
    assert W.rel_err(F32, F64)[0] <= 1e-5
    assert abs(E32 - E64) <= 1e-6 * abs(E64)
    assert np.array_equal(F32, e32.forces(cfg["xyz"], cfg["q"], energy=True)[0])
    # the energy-less kernels are other template instances: same forces to FP32 rounding
    assert W.rel_err(e32.forces(cfg["xyz"], cfg["q"]), F32)[0] <= 1e-6
    em = W.engine_for(cfg, "fp64", mode_flags=L.QEM_DIR_MINIMAGE)
    Fa = em.forces(cfg["xyz"], cfg["q"], terms=L.QEM_TERM_SHORT)
    sh = cfg["xyz"].copy()
    sh[:, 0] = (sh[:, 0] + 123.456) % cfg["L"][0]
    sh[:, 1] = (sh[:, 1] + 654.321) % cfg["L"][1]
    Fb = em.forces(sh, cfg["q"], terms=L.QEM_TERM_SHORT)
    assert W.rel_err(Fb, Fa)[0] <= 1e-10


def test_pair_list_overflow_retry_matches_oracle():
    """Particles packed into a 20 x 20 patch of a 200 x 200 box: the first
    pair-capacity estimate (from the mean density) is ~20 times too small, the
    call overflows, grows the capacity and evaluates again; the forces equal
    the oracle's and a second call repeats them bit for bit."""
    rng = np.random.default_rng(77)
    N, Lb = 1500, (200.0, 200.0, 10.0)
    xyz = np.stack([50 + 20 * rng.random(N), 80 + 20 * rng.random(N), 0.5 + 9 * rng.random(N)], 1)
    q = np.where(np.arange(N) < N // 2, 1.0, -1.0)
    e = Engine(L_box=Lb, alpha=0.1, r_cutoff=10.0, gamma_1=0.5, gamma_2=-0.4, rbe_p=0)
    F = e.forces(xyz, q, terms=L.QEM_TERM_SHORT)
    Fref = O.short_forces(oparams(Lb, 0.1, 10.0, 0.5, -0.4), xyz, q)
    assert W.rel_err(F, Fref)[0] <= 1e-11
    assert np.array_equal(e.forces(xyz, q, terms=L.QEM_TERM_SHORT), F)
