"""Exact (non-random-batch) long range through the C-ABI: every lattice k with
0 < |k| < k_cutoff weighted by exp(-k^2 / 4 alpha) (Force_long.jl:220-233, typos
fixed), against the reference's python exact path (long_exact.json) and the
oracle; per-row weights are the only change to the random-batch kernels."""
import json
import os
import sys

import numpy as np
import pytest

from qem4molly_b200 import _lib as L
from qem4molly_b200 import api
from qem4molly_b200 import workloads as W

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import oracle as O  # noqa: E402

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _engine(Lb, alpha, g_down, g_up, prec="fp64", r_cutoff=1.0):
    return api.Engine(L_box=Lb, alpha=alpha, r_cutoff=r_cutoff, gamma_1=g_down, gamma_2=g_up, rbe_p=0,
                      precision={"fp64": L.QEM_FP64, "fp32": L.QEM_FP32_FIX}[prec])


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-10), ("fp32", 1e-5)])
def test_exact_vs_python_exact_path(prec, tol):
    d = json.load(open(os.path.join(GOLD, "long_exact.json")))
    xyz, q = np.array(d["xyz"]), np.array(d["q"])
    e = _engine(d["L"], d["alpha"], d["gamma_1"], d["gamma_2"], prec)
    assert e.set_kset_exact(d["k_cutoff"]) == d["n_k"]
    F = e.forces(xyz, q, terms=L.QEM_TERM_LONG)
    err, _ = W.rel_err(F, np.array(d["F_long"]))
    assert err <= tol, err


@pytest.fixture(scope="module")
def slab():
    cfg = W.config1()
    k3, w = O.exact_kset(cfg["L"], cfg["alpha"], 1.2)
    p = O.params(cfg["L"], cfg["alpha"], cfg["r_cutoff"], cfg["gamma_down"], cfg["gamma_up"])
    F = O.F_long_weighted(p, cfg["xyz"], cfg["q"], k3, w)
    E = O.energy_long_weighted(p, cfg["xyz"], cfg["q"], k3, w)
    return cfg, k3, w, F, E


@pytest.mark.parametrize("prec,ftol,etol", [("fp64", 1e-9, 1e-10), ("fp32", 1e-5, 1e-5)])
def test_exact_vs_oracle(slab, prec, ftol, etol):
    cfg, k3, w, Fo, Eo = slab
    e = _engine(cfg["L"], cfg["alpha"], cfg["gamma_down"], cfg["gamma_up"], prec, cfg["r_cutoff"])
    assert e.set_kset_exact(1.2) == k3.shape[0] > 1000
    rows, _ = e.get_kset()
    np.testing.assert_array_equal(rows, k3)
    np.testing.assert_array_equal(e.get_kset_weights(), w)
    F, E = e.forces(cfg["xyz"], cfg["q"], terms=L.QEM_TERM_LONG, energy=True)
    err, _ = W.rel_err(F, Fo)
    assert err <= ftol, err
    assert abs(E - Eo) <= etol * abs(Eo), (E, Eo)


def test_uniform_weights_equal_the_random_batch():
    """Weights sum_K / P give the random-batch call bit for bit; set_kset drops the weights."""
    cfg = W.config1()
    e = W.engine_for(cfg, "fp64")
    k3, sum_K = e.get_kset()
    F1 = e.forces(cfg["xyz"], cfg["q"])
    e.set_kset_weighted(k3, np.full(k3.shape[0], sum_K / k3.shape[0]))
    F2 = e.forces(cfg["xyz"], cfg["q"])
    np.testing.assert_array_equal(F1, F2)
    e.set_kset(k3, sum_K)
    assert e.get_kset_weights() is None
    np.testing.assert_array_equal(e.forces(cfg["xyz"], cfg["q"]), F1)


def test_exact_shards_sum_to_the_whole(slab):
    cfg, k3, w, _, _ = slab
    e = _engine(cfg["L"], cfg["alpha"], cfg["gamma_down"], cfg["gamma_up"], "fp64", cfg["r_cutoff"])
    e.set_kset_exact(1.2)
    full = e.forces(cfg["xyz"], cfg["q"], terms=L.QEM_TERM_LONG)
    acc = np.zeros_like(full)
    for r in range(3):
        e.set_shard(r, 3)
        acc += e.forces(cfg["xyz"], cfg["q"], terms=L.QEM_TERM_LONG)
    e.set_shard(0, 1)
    assert np.abs(acc - full).max() <= 1e-12 * np.abs(full).max()


def test_exact_adjoint_vs_fd():
    """qem_backward with the exact k-set against central differences (positions, charges)."""
    cfg = W.config3(N=300)
    rng = np.random.default_rng(4)
    e = _engine(cfg["L"], cfg["alpha"], cfg["gamma_down"], cfg["gamma_up"], "fp64", cfg["r_cutoff"])
    assert e.set_kset_exact(0.5) > 40
    xyz, q = cfg["xyz"].copy(), cfg["q"].copy()
    gF = rng.normal(size=xyz.shape)
    gE, h, terms = 0.7, 1e-4, L.QEM_TERM_LONG
    gx, gq, _ = e.backward(xyz, q, gF, gE, terms=terms)
    z = xyz[:, 2]
    gaps = np.array([np.min(np.abs(np.delete(z, i) - z[i])) for i in range(len(z))])

    def L_of(x, qq):
        F, E = e.forces(x, qq, terms=terms, energy=True)
        return F, E

    sx, sq = np.sqrt(np.mean(gx ** 2)), np.sqrt(np.mean(gq ** 2))
    for i in [int(i) for i in np.argsort(-gaps)[:5]]:
        for a in range(3):
            xp, xm = xyz.copy(), xyz.copy()
            xp[i, a] += h
            xm[i, a] -= h
            (Fp, Ep), (Fm, Em) = L_of(xp, q), L_of(xm, q)
            fd = (np.sum(gF * (Fp - Fm)) + gE * (Ep - Em)) / (2 * h)
            assert abs(fd - gx[i, a]) <= 2e-6 * (abs(fd) + sx), (i, a, fd, gx[i, a])
        qp, qm = q.copy(), q.copy()
        qp[i] += h
        qm[i] -= h
        (Fp, Ep), (Fm, Em) = L_of(xyz, qp), L_of(xyz, qm)
        fd = (np.sum(gF * (Fp - Fm)) + gE * (Ep - Em)) / (2 * h)
        assert abs(fd - gq[i]) <= 2e-6 * (abs(fd) + sq), (i, fd, gq[i])


def test_qem_long_rbe_mode_false(slab):
    cfg, k3, _, Fo, _ = slab
    inter = api.QEM_long(cfg["L"], k_cutoff=1.2, gamma_1=cfg["gamma_down"], gamma_2=cfg["gamma_up"],
                         alpha=cfg["alpha"], rbe_mode=False)
    assert inter.n_k == k3.shape[0]
    F = api.forces(inter, api.System(coords=cfg["xyz"], charges=cfg["q"]))
    err, _ = W.rel_err(F, Fo)
    assert err <= 1e-9, err
