"""Batches of independent systems (qem_batch_*): batched forces equal the
per-system calls (bit for bit on the stream pool; to 1e-14 in the fused
phases, whose kernels run the same per-block code compiled into other
kernels, where FP64 multiply-adds may contract differently); the
graph-replayed velocity-Verlet run matches an eager host loop over the
per-system calls; the autotuner's choice keeps the results.  Systems from
the many-slab workload (N ~ U[200, 5000], Lz ~ U[5, 20], density 0.01,
gamma pairs ~ U(-0.95, 0.95)^2, P = 200)."""

FUSED_TOL = 1e-14  # fused phases against the same system's own call (max |dF| / rms |F|)


def _close(F, ref, tol=FUSED_TOL):
    return float(np.abs(F - ref).max() / np.sqrt(np.mean(ref ** 2))) <= tol
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
    fused = b.mode()["mode"] == "fused"
    assert fused == (prec == "fp32")
    for c, e, o, n in zip(cfgs, engines, b.off, N):
        own = e.forces(c["xyz"], c["q"])
        assert _close(Fb[o:o + n], own) if fused else np.array_equal(Fb[o:o + n], own)


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


# ---------------------------------------------------------------- fused phases
def _batch_F(b, x, q):
    import torch

    F = torch.empty_like(x)
    b.forces(x, q, F)
    F.zero_()
    b.forces(x, q, F)
    b.check()
    return F.cpu().numpy()


def test_fused_batch_runs_fused_and_pool_agrees():
    """FP32+fix systems of the many-slab workload qualify for the fused phases
    (16 or 17 launches per evaluation); forcing the stream pool gives the same
    forces (same per-block code, same k-slices) to FUSED_TOL."""
    cfgs, engines, N, x, q = _setup(16, "fp32")
    b = Batch(engines, N)
    Ff = _batch_F(b, x, q)
    m = b.mode()
    assert m["mode"] == "fused" and m["launches"] in (16, 17) and m["why"] == "", m
    b.set_mode(L.QEM_BATCH_POOL)
    Fp = _batch_F(b, x, q)
    assert b.mode()["mode"] == "pool"
    assert _close(Ff, Fp)


def test_fused_batch_tilings_agree():
    """Other fused tilings (at most 1 or 2 k-slices per system, largest
    system first) change only the order of the k-slice sums; shorter chunks
    regroup the FP32 structure sums as well."""
    cfgs, engines, N, x, q = _setup(10, "fp32", seed=77)
    b = Batch(engines, N)
    ref = _batch_F(b, x, q)
    for ks, order, chunk in ((1, 0, 0), (2, 1, 0), (0, 1, 0), (0, 0, 128), (2, 1, 64)):
        b.set_mode(L.QEM_BATCH_FUSED, ks, order, chunk)
        F = _batch_F(b, x, q)
        assert b.mode()["chunk"] == (chunk or 512)
        # other chunks regroup the FP32 structure sums (FP32 rounding, ~1e-7)
        assert W.rel_err(F, ref)[0] <= (1e-12 if chunk == 0 else 1e-6), (ks, order, chunk)
        if ks == 0 and chunk == 0:
            assert np.array_equal(F, ref)


def test_fused_batch_vs_oracle_and_fp64():
    """Fused FP32+fix forces against the FP64 oracle on the three thinnest
    slabs of the batch (short range over all pairs and self terms, long range
    with each system's k-set), and against each system's FP64 GPU evaluation
    on the same k-set for every slab, to 1e-5 relative.  (The oracle restates
    the reference's long-range running sums, Force_long.jl:97-98, which lose
    digits like e^{k L_z}: at L_z = 19.9 its long range is 4e-5 from the GPU
    FP64 path while the short ranges agree to 3e-16; the thick slabs are
    therefore checked against FP64 on the GPU.)"""
    import oracle as O

    cfgs, engines, N, x, q = _setup(8, "fp32", seed=31)
    b = Batch(engines, N)
    Fb = _batch_F(b, x, q)
    assert b.mode()["mode"] == "fused"
    thin = sorted(range(len(cfgs)), key=lambda s: cfgs[s]["L"][2])[:3]
    for s in range(len(cfgs)):
        c, e, o, n = cfgs[s], engines[s], b.off[s], N[s]
        k3, sK = e.get_kset()
        e64 = W.engine_for(c, "fp64")
        e64.set_kset(k3, sK)
        F64 = e64.forces(c["xyz"], c["q"])
        e64.close()
        assert W.rel_err(Fb[o:o + n], F64)[0] <= 1e-5, s
        if s in thin:
            assert c["L"][2] <= 12.0
            p = O.params(c["L"], c["alpha"], c["r_cutoff"], c["gamma_down"], c["gamma_up"], accuracy=c["accuracy"],
                         N_t=c["N_t"])
            Fo = O.short_forces(p, c["xyz"], c["q"]) + O.F_long(p, c["xyz"], c["q"], k3, sK)
            assert W.rel_err(F64, Fo)[0] <= 1e-9, s
            assert W.rel_err(Fb[o:o + n], Fo)[0] <= 1e-5, s


def _batch_counter(e):
    import ctypes as C

    n = C.c_uint64()
    assert e._lib.qem_kset_batch(e._h, C.byref(n)) == 0
    return n.value


def test_fused_batch_resamples_every_call():
    """With QEM_RESAMPLE_KSET every fused evaluation draws each system's next
    batch on the device: evaluation n of the batch equals the system's own
    call n from the same seed (replayed afterwards on the same handles)."""
    import torch

    cfgs = W.config4(seed=55, n_systems=6)
    engines = [W.engine_for(c, "fp32", mode_flags=L.QEM_RESAMPLE_KSET, seed=300 + i) for i, c in enumerate(cfgs)]
    N = [c["N"] for c in cfgs]
    dev = torch.device("cuda", 0)
    x = torch.tensor(np.concatenate([c["xyz"] for c in cfgs]), device=dev)
    q = torch.tensor(np.concatenate([c["q"] for c in cfgs]), device=dev)
    b = Batch(engines, N)
    F = torch.empty_like(x)
    b.forces(x, q, F)  # sizing pass: batch 0 of every system
    assert b.mode()["mode"] == "fused"
    got, rows = [], []
    for n in (1, 2):
        b.forces(x, q, F)
        b.check()
        got.append(F.cpu().numpy().copy())
        rows.append([e.get_kset()[0].copy() for e in engines])
        assert [_batch_counter(e) for e in engines] == [n + 1] * len(engines)
    for i, (c, e, o, k) in enumerate(zip(cfgs, engines, b.off, N)):
        e.sample_kset(300 + i, c["P"])  # batch counter back to 0
        own = [e.forces(c["xyz"], c["q"]) for _ in range(3)]
        for n in (1, 2):
            assert _close(got[n - 1][o:o + k], own[n]), (i, n)
        e.sample_kset(300 + i, c["P"])
        for n in range(3):
            e.forces(c["xyz"], c["q"])
            if n >= 1:
                assert np.array_equal(e.get_kset()[0], rows[n - 1][i])


def test_fused_batch_md_draws_a_batch_per_step():
    import torch

    cfgs = W.config4(seed=56, n_systems=4)
    engines = [W.engine_for(c, "fp32", mode_flags=L.QEM_RESAMPLE_KSET, seed=400 + i) for i, c in enumerate(cfgs)]
    N = [c["N"] for c in cfgs]
    dev = torch.device("cuda", 0)
    x = torch.tensor(np.concatenate([c["xyz"] for c in cfgs]), device=dev)
    q = torch.tensor(np.concatenate([c["q"] for c in cfgs]), device=dev)
    v = torch.zeros_like(x)
    F = torch.empty_like(x)
    b = Batch(engines, N)
    b.md(10, 1e-3, x, v, q, F)
    assert b.mode()["mode"] == "fused"
    c0 = [_batch_counter(e) for e in engines]
    b.md(25, 1e-3, x, v, q, F)
    assert [_batch_counter(e) - c for e, c in zip(engines, c0)] == [26] * 4  # 1 evaluation + 25 steps
    assert np.isfinite(x.cpu().numpy()).all()


def test_fused_batch_autotune_keeps_results():
    import torch

    cfgs, engines, N, x, q = _setup(16, "fp32", seed=12)
    b = Batch(engines, N)
    ref = _batch_F(b, x, q)
    w, ms = b.autotune(x, q, torch.empty_like(x))
    assert ms > 0 and 0 <= w <= 16
    assert (b.mode()["mode"] == "fused") == (w == 0)
    F = _batch_F(b, x, q)
    assert W.rel_err(F, ref)[0] <= (1e-12 if b.mode()["chunk"] == 512 else 1e-6)


def test_fused_batch_with_walls():
    """Substrate_LJ walls are fused into the gather of the fused phases as in
    the systems' own calls (config-1-like slabs with walls at z = 0 and L_z)."""
    import torch

    from qem4molly_b200.api import Engine, Substrate_LJ

    rng = np.random.default_rng(23)
    cfgs, engines = [], []
    for i, n in enumerate((150, 400, 900)):
        Lxy = float(np.sqrt(n / 0.01))
        xyz = np.stack([rng.random(n) * Lxy, rng.random(n) * Lxy, 0.5 + 9.0 * rng.random(n)], 1)
        q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
        walls = [Substrate_LJ(cutoff=1.0, sigma=1.0, eps=1.0, sub_pos=0.0, direction=1),
                 Substrate_LJ(cutoff=1.0, sigma=1.0, eps=1.0, sub_pos=10.0, direction=-1)]
        e = Engine(L_box=(Lxy, Lxy, 10.0), alpha=0.1, r_cutoff=10.0, gamma_1=0.6, gamma_2=-0.8, rbe_p=60,
                   walls=walls, precision=L.QEM_FP32_FIX)
        e.sample_kset(70 + i, 60)
        cfgs.append(dict(xyz=xyz, q=q, N=n))
        engines.append(e)
    x = torch.tensor(np.concatenate([c["xyz"] for c in cfgs]), device="cuda")
    q = torch.tensor(np.concatenate([c["q"] for c in cfgs]), device="cuda")
    b = Batch(engines, [c["N"] for c in cfgs])
    Fb = _batch_F(b, x, q)
    assert b.mode()["mode"] == "fused"
    for c, e, o in zip(cfgs, engines, b.off):
        own = e.forces(c["xyz"], c["q"])
        assert _close(Fb[o:o + c["N"]], own)
        no_walls = e.forces(c["xyz"], c["q"], terms=L.QEM_TERM_SHORT | L.QEM_TERM_LONG)
        assert np.abs(own - no_walls).max() > 0  # the walls act on these slabs


def test_fused_batch_recovers_from_a_pair_list_overflow():
    """Positions whose pair list outgrows the capacity sized on the first call:
    check() reports QEM_ERR_NB_OVERFLOW, and the next batch call sizes every
    system again and equals the systems' own calls."""
    import torch

    cfgs, engines, N, x, q = _setup(6, "fp32", seed=41)
    b = Batch(engines, N)
    F = torch.empty_like(x)
    b.forces(x, q, F)
    assert b.mode()["mode"] == "fused"
    # squeeze system 2 into a quarter of its box in x and y: ~16x the pairs
    o, n = b.off[2], N[2]
    xs = x.clone()
    xs[o:o + n, :2] *= 0.25
    b.forces(xs, q, F)
    with pytest.raises(L.QemError) as err:
        b.check()
    assert err.value.status == 4  # QEM_ERR_NB_OVERFLOW
    b.forces(xs, q, F)  # sizes every system again (synchronously)
    b.forces(xs, q, F)
    b.check()
    assert b.mode()["mode"] == "fused"
    Fb = F.cpu().numpy()
    xh = xs.cpu().numpy()
    for c, e, oo, nn in zip(cfgs, engines, b.off, N):
        assert _close(Fb[oo:oo + nn], e.forces(xh[oo:oo + nn], c["q"]))


@pytest.mark.parametrize("mode", [L.QEM_BATCH_FUSED, L.QEM_BATCH_POOL])
def test_batch_follows_a_changed_kset(mode):
    """A new k-set fed to one handle between batch calls is sized and uploaded
    by the next batch call (fused phases and stream pool alike), whose forces
    then equal the systems' own calls with their current k-sets."""
    import torch

    cfgs, engines, N, x, q = _setup(5, "fp32", seed=43)
    b = Batch(engines, N)
    b.set_mode(mode)
    _batch_F(b, x, q)
    other = W.engine_for(cfgs[3], "fp32", seed=999)
    k3, sK = other.get_kset()
    engines[3].set_kset(k3, sK)
    Fb = _batch_F(b, x, q)
    assert b.mode()["mode"] == ("fused" if mode == L.QEM_BATCH_FUSED else "pool")
    assert np.array_equal(engines[3].get_kset()[0], k3)
    for c, e, o, n in zip(cfgs, engines, b.off, N):
        own = e.forces(c["xyz"], c["q"])
        assert _close(Fb[o:o + n], own) if mode == L.QEM_BATCH_FUSED else np.array_equal(Fb[o:o + n], own)


def test_batch_mode_arguments():
    """Bad modes, k-slice counts, orders and chunk lengths are refused; a
    fused request for a batch that cannot run fused (FP64 systems) fails at
    the next batch call and names the reason; the pool request runs."""
    import torch

    cfgs, engines, N, x, q = _setup(3, "fp64", seed=44)
    b = Batch(engines, N)
    for args in ((7, 0, 0, 0), (L.QEM_BATCH_FUSED, -1, 0, 0), (L.QEM_BATCH_FUSED, 0, 2, 0),
                 (L.QEM_BATCH_FUSED, 0, 0, 100), (L.QEM_BATCH_FUSED, 0, 0, 16)):
        with pytest.raises(L.QemError) as err:
            b.set_mode(*args)
        assert err.value.status == 1, args
    b.set_mode(L.QEM_BATCH_FUSED)
    F = torch.empty_like(x)
    with pytest.raises(L.QemError) as err:
        b.forces(x, q, F)
        b.forces(x, q, F)
    assert "QEM_FP32_FIX" in str(err.value)
    b.set_mode(L.QEM_BATCH_POOL)
    Fb = _batch_F(b, x, q)
    assert b.mode()["mode"] == "pool" and b.mode()["launches"] == -1
    for c, e, o, n in zip(cfgs, engines, b.off, N):
        assert np.array_equal(Fb[o:o + n], e.forces(c["xyz"], c["q"]))
