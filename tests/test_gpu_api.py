"""The Molly-facing Python mirror (qem4molly_b200.api) against the FP64 oracle,
on config 1 (N = 100, Lx = Ly = 100, Lz = 10, gamma_up = 0.95,
gamma_down = -0.95, alpha = 0.1, r_c = 10, N_t = 30, P = 100, LJ walls):

* QEM_short + forces / potential_energy (QEM_short.jl:19-59);
* QEM_long(rbe_mode=True) with its default per-call random batch
  (Force_long.jl:235): every call's batch is read back and fed to the oracle;
  consecutive calls draw different batches, batch n is the sampler's batch n
  (qem_draw_kset) in both precisions, also through the recorded-graph path;
* QEM_inter (Quasi_Ewald_Method.jl:3-24) in both modes;
* forces(Substrate_LJ) (Substrate_LJ.jl:24-46).

Tolerances: FP64 forces <= 1e-10 relative L2 (short range 1e-11), energies
<= 1e-10 relative; FP32+fix forces <= 1e-5 (the metric's bound).
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from qem4molly_b200 import _lib as L
from qem4molly_b200 import api
from qem4molly_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cfg():
    return W.config1()


def oparams(c, alpha=None, rc=None):
    return O.params(c["L"], c["alpha"] if alpha is None else alpha, c["r_cutoff"] if rc is None else rc,
                    c["gamma_down"], c["gamma_up"], accuracy=c["accuracy"], N_t=c["N_t"])


def system(c):
    return api.System(coords=c["xyz"].copy(), charges=c["q"].copy())


def draw_rows(params, seed, n, P):
    k3 = np.zeros((P, 3))
    sK = C.c_double()
    assert L.load().qem_draw_kset(C.byref(params), seed, n, 0, P, k3.ctypes.data_as(C.POINTER(C.c_double)),
                                  C.byref(sK)) == 0
    return k3, sK.value


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-11), ("fp32", 1e-5)])
def test_qem_short_forces_and_energy(cfg, precision, tol):
    inter = api.QEM_short(cfg["L"], cfg["r_cutoff"], cfg["alpha"], gamma_1=cfg["gamma_down"],
                          gamma_2=cfg["gamma_up"], accuracy=cfg["accuracy"], N_t=cfg["N_t"], precision=precision)
    sys_ = system(cfg)
    F = api.forces(inter, sys_)
    p = oparams(cfg)
    assert W.rel_err(F, O.short_forces(p, cfg["xyz"], cfg["q"]))[0] <= tol
    assert inter.n_steps == 1
    E = api.potential_energy(inter, sys_)
    assert np.isclose(E, O.energy_short(p, cfg["xyz"], cfg["q"]), rtol=1e-10 if precision == "fp64" else 1e-5)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("fp32", 1e-5)])
def test_qem_long_draws_a_fresh_batch_every_call(cfg, precision, tol):
    inter = api.QEM_long(cfg["L"], gamma_1=cfg["gamma_down"], gamma_2=cfg["gamma_up"], accuracy=cfg["accuracy"],
                         alpha=cfg["alpha"], rbe_p=cfg["P"], precision=precision, seed=2024)
    assert inter.rbe_mode
    sys_ = system(cfg)
    p = oparams(cfg)
    prev = None
    for n in range(3):
        F = api.forces(inter, sys_)
        k3, sK = inter.engine.get_kset()
        rows, sK_ref = draw_rows(inter.engine.params, 2024, n, cfg["P"])
        np.testing.assert_array_equal(k3, rows)  # call n used batch n of the seed
        assert sK == sK_ref
        assert W.rel_err(F, O.F_long(p, cfg["xyz"], cfg["q"], k3, sK))[0] <= tol
        if prev is not None:
            assert not np.array_equal(prev, k3)
        prev = k3
    # the energy call draws the next batch too; its value is the oracle's for that batch
    E = api.potential_energy(inter, sys_)
    k3, sK = inter.engine.get_kset()
    np.testing.assert_array_equal(k3, draw_rows(inter.engine.params, 2024, 3, cfg["P"])[0])
    assert np.isclose(E, O.energy_long(p, cfg["xyz"], cfg["q"], k3, sK), rtol=1e-10 if precision == "fp64" else 1e-5)
    # resample=False keeps one batch
    fixed = api.QEM_long(cfg["L"], gamma_1=cfg["gamma_down"], gamma_2=cfg["gamma_up"], alpha=cfg["alpha"],
                         rbe_p=cfg["P"], precision=precision, seed=2024, resample=False)
    a = api.forces(fixed, sys_)
    assert np.array_equal(a, api.forces(fixed, sys_))


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("fp32", 1e-5)])
def test_resampling_through_recorded_graph_and_device_memory(cfg, precision, tol):
    """Repeated device-memory calls replay a recorded graph; the batch counter
    in device memory still gives call n batch n."""
    import torch

    e = W.engine_for(cfg, precision, mode_flags=L.QEM_RESAMPLE_KSET, seed=77)
    x = torch.tensor(cfg["xyz"], dtype=torch.float64, device="cuda")
    q = torch.tensor(cfg["q"], dtype=torch.float64, device="cuda")
    F = torch.empty_like(x)
    p = oparams(cfg)
    Fo = O.short_forces(p, cfg["xyz"], cfg["q"]) + O.lj_two_walls(cfg["xyz"], cfg["walls"])[0]
    for n in range(6):
        e.forces_device(x, q, F)
        torch.cuda.synchronize()
        if n >= 2:
            assert e.counts()["launches"] > 0
        nb = C.c_uint64()
        assert L.load().qem_kset_batch(e._h, C.byref(nb)) == 0 and nb.value == n + 1
        k3, sK = e.get_kset()
        np.testing.assert_array_equal(k3, draw_rows(e.params, 77, n, cfg["P"])[0])
        ref = Fo + O.F_long(p, cfg["xyz"], cfg["q"], k3, sK)
        assert W.rel_err(F.cpu().numpy(), ref)[0] <= tol, n
    # qem_sample_kset restarts the batches
    e.sample_kset(77, cfg["P"])
    e.forces_device(x, q, F)
    np.testing.assert_array_equal(e.get_kset()[0], draw_rows(e.params, 77, 0, cfg["P"])[0])


def test_resampled_backward_uses_the_latest_batch(cfg):
    e = W.engine_for(cfg, "fp64", mode_flags=L.QEM_RESAMPLE_KSET, seed=5)
    for _ in range(2):
        e.forces(cfg["xyz"], cfg["q"], terms=L.QEM_TERM_LONG)
    k3, sK = e.get_kset()
    gx, gq, gg = e.backward(cfg["xyz"], cfg["q"], None, 1.0, terms=L.QEM_TERM_LONG)
    fixed = W.engine_for(cfg, "fp64")
    fixed.set_kset(k3, sK)
    gx2, gq2, gg2 = fixed.backward(cfg["xyz"], cfg["q"], None, 1.0, terms=L.QEM_TERM_LONG)
    np.testing.assert_array_equal(gx, gx2)
    np.testing.assert_array_equal(gq, gq2)
    np.testing.assert_array_equal(gg, gg2)
    # the backward does not advance the batches
    nb = C.c_uint64()
    assert L.load().qem_kset_batch(e._h, C.byref(nb)) == 0 and nb.value == 2


def test_resampled_shards_sum_to_the_whole(cfg):
    """Each rank draws its own rows of the same batch: the W shares of call n
    sum to the unsharded call n."""
    c = W.config2(N=3000, seed=4)
    whole = W.engine_for(c, "fp64", mode_flags=L.QEM_RESAMPLE_KSET, seed=9)
    parts = []
    for r in range(3):
        e = W.engine_for(c, "fp64", mode_flags=L.QEM_RESAMPLE_KSET, seed=9)
        e.set_shard(r, 3)
        parts.append(e)
    for _ in range(2):
        F = whole.forces(c["xyz"], c["q"])
        Fs = sum(e.forces(c["xyz"], c["q"]) for e in parts)
        assert W.rel_err(Fs, F)[0] <= 1e-12


@pytest.mark.parametrize("rbe_mode", [True, False])
def test_qem_inter(cfg, rbe_mode):
    N = len(cfg["q"])
    s = 1.0
    short, long = api.QEM_inter(N, cfg["L"], s=s, rbe_mode=rbe_mode, rbe_p=50, gamma_1=cfg["gamma_down"],
                                gamma_2=cfg["gamma_up"], seed=3)
    Lx, Ly, _ = cfg["L"]
    alpha = N / (Lx * Ly) if rbe_mode else np.sqrt(N) / (Lx * Ly)  # Quasi_Ewald_Method.jl:6, 14
    assert np.isclose(short.alpha, alpha) and np.isclose(long.alpha, alpha)
    assert np.isclose(short.r_cutoff, s / np.sqrt(alpha)) and np.isclose(long.k_cutoff, 2 * s * np.sqrt(alpha))
    assert long.rbe_mode == rbe_mode
    sys_ = system(cfg)
    p = oparams(cfg, alpha=alpha, rc=s / np.sqrt(alpha))
    Fs = api.forces(short, sys_)
    assert W.rel_err(Fs, O.short_forces(p, cfg["xyz"], cfg["q"]))[0] <= 1e-11
    Fl = api.forces(long, sys_)
    if rbe_mode:
        k3, sK = long.engine.get_kset()
        Fo = O.F_long(p, cfg["xyz"], cfg["q"], k3, sK)
    else:
        k3, w = O.exact_kset(cfg["L"][:2], alpha, 2 * s * np.sqrt(alpha))
        Fo = O.F_long_weighted(p, cfg["xyz"], cfg["q"], k3, w)
    assert W.rel_err(Fl, Fo)[0] <= 1e-10


def test_forces_substrate_lj(cfg):
    sys_ = system(cfg)
    for w in cfg["walls"]:
        F = api.forces(api.Substrate_LJ(**w), sys_)
        Fo, bad = O.lj_forces(cfg["xyz"], w["cutoff"], w["sigma"], w["eps"], w["sub_pos"], w["direction"])
        assert bad == 0
        assert np.allclose(F, Fo, rtol=1e-13, atol=1e-14 * max(np.abs(Fo).max(), 1e-300))
    with pytest.raises(TypeError):
        api.potential_energy(api.Substrate_LJ(), sys_)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_resampling_with_the_constants_on_their_own_stream(precision):
    """Above 8192 particles (and whenever the energy is asked for) the per-k
    constants, and with per-call batches the draw of the batch, run on a
    stream of their own beside the z order, and the chunk totals wait for
    them.  On a 2e4-particle slab, call n must still use batch n of the seed,
    through the recorded graph and through an ordinary call with the energy,
    and give the forces (and energy) of a handle fed batch n explicitly."""
    import torch

    cfg = W.config2(N=20_000, seed=11)
    e = W.engine_for(cfg, precision, mode_flags=L.QEM_RESAMPLE_KSET, seed=31)
    ref = W.engine_for(cfg, precision)
    x = torch.tensor(cfg["xyz"], dtype=torch.float64, device="cuda")
    q = torch.tensor(cfg["q"], dtype=torch.float64, device="cuda")
    F = torch.empty_like(x)
    for n in range(5):
        e.forces_device(x, q, F)
        torch.cuda.synchronize()
        rows, sK = draw_rows(e.params, 31, n, cfg["P"])
        np.testing.assert_array_equal(e.get_kset()[0], rows)
        ref.set_kset(rows, sK)
        assert W.rel_err(F.cpu().numpy(), ref.forces(cfg["xyz"], cfg["q"]))[0] <= 1e-13, n
    Fe, E = e.forces(cfg["xyz"], cfg["q"], energy=True)
    rows, sK = draw_rows(e.params, 31, 5, cfg["P"])
    np.testing.assert_array_equal(e.get_kset()[0], rows)
    ref.set_kset(rows, sK)
    Fr, Er = ref.forces(cfg["xyz"], cfg["q"], energy=True)
    assert W.rel_err(Fe, Fr)[0] <= 1e-13 and abs(E - Er) <= 1e-13 * abs(Er)
    e.close()
    ref.close()
