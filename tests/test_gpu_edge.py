"""Edge cases of the force path against the FP64 oracle: an empty system, a
single particle (self terms and the long range of one charge), a pair with
the same (x, y) (rho = 0, Force_short.jl:46), a pair exactly at the cutoff
(rho^2 == r_c^2 is a pair: the reference's neighbour test is <=), an empty
k-set (the k = 0 term alone), zero charges, no dielectric contrast, and
ragged batches (systems of 1 .. 2500 particles, and one with none).
FP64 to 1e-10 (1e-9 for the long range), FP32+fix to 1e-5, relative L2."""
import numpy as np
import pytest

import oracle as O
from qem4molly_b200 import _lib as L
from qem4molly_b200 import workloads as W
from qem4molly_b200.api import Batch, Engine

pytestmark = pytest.mark.gpu

BOX = (40.0, 40.0, 10.0)
TOL = {"fp64": 1e-10, "fp32": 1e-5}


def _engine(prec, g_down=-0.7, g_up=0.9, P=24, seed=5):
    e = Engine(L_box=BOX, alpha=0.1, r_cutoff=10.0, gamma_1=g_down, gamma_2=g_up, rbe_p=P,
               precision={"fp64": L.QEM_FP64, "fp32": L.QEM_FP32_FIX}[prec])
    e.sample_kset(seed, P)
    return e


def _oracle(xyz, q, e, g_down=-0.7, g_up=0.9):
    p = O.params(BOX, 0.1, 10.0, g_down, g_up)
    k3, sK = e.get_kset()
    return O.short_forces(p, xyz, q), O.F_long(p, xyz, q, k3, sK)


def _err(F, ref):
    n = np.linalg.norm(ref)
    return float(np.linalg.norm(F - ref) / n) if n > 0 else float(np.abs(F).max())


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_empty_system(prec):
    e = _engine(prec)
    F, E = e.forces(np.zeros((0, 3)), np.zeros(0), energy=True)
    assert F.shape == (0, 3) and E == 0.0


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_single_particle(prec):
    e = _engine(prec)
    xyz, q = np.array([[12.5, 30.25, 3.2]]), np.array([0.7])
    Fs, Fl = _oracle(xyz, q, e)
    assert np.all(Fs[:, :2] == 0.0) and abs(Fs[0, 2]) > 0  # the self image force is along z
    assert _err(e.forces(xyz, q, terms=L.QEM_TERM_SHORT), Fs) <= TOL[prec]
    assert _err(e.forces(xyz, q, terms=L.QEM_TERM_LONG), Fl) <= max(TOL[prec], 1e-9)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_pair_with_the_same_xy(prec):
    e = _engine(prec)
    xyz, q = np.array([[7.0, 9.0, 2.0], [7.0, 9.0, 7.5]]), np.array([1.0, -1.0])
    Fs, Fl = _oracle(xyz, q, e)
    F = e.forces(xyz, q, terms=L.QEM_TERM_SHORT)
    assert np.all(F[:, :2] == 0.0)
    assert _err(F, Fs) <= TOL[prec]
    assert _err(e.forces(xyz, q, terms=L.QEM_TERM_LONG), Fl) <= max(TOL[prec], 1e-9)


def test_pair_exactly_at_the_cutoff():
    e = _engine("fp64")
    p = O.params(BOX, 0.1, 10.0, -0.7, 0.9)
    at = np.array([[5.0, 5.0, 3.0], [15.0, 5.0, 6.0]])        # rho = 10 exactly
    past = np.array([[5.0, 5.0, 3.0], [15.000001, 5.0, 6.0]])
    assert e.pair_list(at).shape[0] == 1 and O.pairs(p, at).shape[0] == 1
    assert e.pair_list(past).shape[0] == 0 and O.pairs(p, past).shape[0] == 0
    q = np.array([1.0, -1.0])
    for xyz in (at, past):
        assert _err(e.forces(xyz, q, terms=L.QEM_TERM_SHORT), O.short_forces(p, xyz, q)) <= 1e-10


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_empty_kset_leaves_the_k0_term(prec):
    e = _engine(prec)
    cfg = W.config1()
    xyz, q = cfg["xyz"] * np.array([0.4, 0.4, 1.0]), cfg["q"]
    e.set_kset(np.zeros((0, 3)), 0.0)
    assert e.get_kset()[0].shape == (0, 3)
    F = e.forces(xyz, q, terms=L.QEM_TERM_LONG)
    Fo = O.F_long(O.params(BOX, 0.1, 10.0, -0.7, 0.9), xyz, q, np.zeros((0, 3)), 0.0)
    assert np.all(F[:, :2] == 0.0) and np.all(Fo[:, :2] == 0.0)
    assert _err(F, Fo) <= 1e-12


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_zero_charges_give_zero_forces(prec):
    e = _engine(prec)
    cfg = W.config1()
    xyz = cfg["xyz"] * np.array([0.4, 0.4, 1.0])
    F, E = e.forces(xyz, np.zeros(len(xyz)), terms=L.QEM_TERM_SHORT | L.QEM_TERM_LONG, energy=True)
    assert np.all(F == 0.0) and E == 0.0


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_no_dielectric_contrast(prec):
    e = _engine(prec, 0.0, 0.0)
    cfg = W.config1()
    xyz, q = cfg["xyz"] * np.array([0.4, 0.4, 1.0]), cfg["q"]
    Fs, Fl = _oracle(xyz, q, e, 0.0, 0.0)
    F = e.forces(xyz, q, terms=L.QEM_TERM_SHORT | L.QEM_TERM_LONG)
    assert _err(F, Fs + Fl) <= max(TOL[prec], 1e-9)


def _ragged(Ns, seed):
    import torch

    rng = np.random.default_rng(seed)
    cfgs = []
    for n in Ns:
        Lxy = max(30.0, float(np.sqrt(max(n, 1) / 0.01)))
        xyz = np.stack([rng.random(n) * Lxy, rng.random(n) * Lxy, 0.5 + 9.0 * rng.random(n)], 1)
        q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
        cfgs.append(dict(L=(Lxy, Lxy, 10.0), xyz=xyz, q=q, N=n))
    engines = []
    for i, c in enumerate(cfgs):
        e = Engine(L_box=c["L"], alpha=0.1, r_cutoff=10.0, gamma_1=-0.5, gamma_2=0.8, rbe_p=40,
                   precision=L.QEM_FP32_FIX)
        e.sample_kset(60 + i, 40)
        engines.append(e)
    dev = torch.device("cuda", 0)
    x = torch.tensor(np.concatenate([c["xyz"] for c in cfgs]).reshape(-1, 3), device=dev)
    q = torch.tensor(np.concatenate([c["q"] for c in cfgs]), device=dev)
    return cfgs, engines, x, q


@pytest.mark.parametrize("Ns,mode", [((1, 2, 37, 300, 2500), "fused"), ((5, 0, 400), "pool")])
def test_ragged_batches(Ns, mode):
    """Systems of very different sizes in one batch equal their own calls;
    a system with no particles sends the batch to the stream pool."""
    import torch

    cfgs, engines, x, q = _ragged(Ns, 17)
    b = Batch(engines, [c["N"] for c in cfgs])
    F = torch.empty_like(x)
    b.forces(x, q, F)
    F.zero_()
    b.forces(x, q, F)
    b.check()
    m = b.mode()
    assert m["mode"] == mode, m
    if mode == "pool":
        assert "system 1" in m["why"]
    Fb = F.cpu().numpy()
    for c, e, o in zip(cfgs, engines, b.off):
        n = c["N"]
        own = e.forces(c["xyz"], c["q"])
        if n == 0:
            continue
        scale = max(float(np.sqrt(np.mean(own ** 2))), 1e-300)
        assert float(np.abs(Fb[o:o + n] - own).max()) / scale <= (1e-14 if mode == "fused" else 0.0)
