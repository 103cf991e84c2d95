"""Equal-z ties in the long range (QEM_EQUAL_Z_TIES): tied particles are neither
below nor above each other in the z-ordered sums (python_lib equal_cell,
Sigma_Gamma_func_njit.py:168-281).  Against the reference's own sums with
equal_cell groups (long_ties.json) and the oracle's group-exclusive restatement;
the energy and untied systems do not change; the adjoint against central
differences in the directions that keep the ties."""
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


def _engine(Lb, alpha, g_down, g_up, k3, sum_K, prec="fp64", ties=True):
    e = api.Engine(L_box=Lb, alpha=alpha, r_cutoff=min(Lb[0], Lb[1]) / 4, gamma_1=g_down, gamma_2=g_up, rbe_p=0,
                   mode_flags=L.QEM_EQUAL_Z_TIES if ties else 0,
                   precision={"fp64": L.QEM_FP64, "fp32": L.QEM_FP32_FIX}[prec])
    e.set_kset(k3, sum_K)
    return e


def _k3(ks):
    ks = np.asarray(ks)
    return np.concatenate([ks, np.hypot(ks[:, 0], ks[:, 1])[:, None]], 1)


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-10), ("fp32", 1e-5)])
def test_ties_vs_python_equal_cell(prec, tol):
    d = json.load(open(os.path.join(GOLD, "long_ties.json")))
    xyz, q = np.array(d["xyz"]), np.array(d["q"])
    Fr = np.array(d["F_long"])
    e = _engine(d["L"], 1.0, d["gamma_1"], d["gamma_2"], _k3(d["kset"]), d["sum_K"], prec)
    F = e.forces(xyz, q, terms=L.QEM_TERM_LONG)
    assert W.rel_err(F, Fr)[0] <= tol
    e0 = _engine(d["L"], 1.0, d["gamma_1"], d["gamma_2"], _k3(d["kset"]), d["sum_K"], prec, ties=False)
    assert W.rel_err(e0.forces(xyz, q, terms=L.QEM_TERM_LONG), Fr)[0] > 0.05


def _tied_slab(N=2000, levels=20, seed=3):
    cfg = W.config3(N=N, seed=seed)
    rng = np.random.default_rng(seed)
    cfg["xyz"][:, 2] = rng.choice(np.linspace(0.6, 9.4, levels), N)
    return cfg


@pytest.mark.parametrize("N,levels", [(2000, 20), (6000, 60), (6000, 12)])
@pytest.mark.parametrize("prec,ftol", [("fp64", 1e-9), ("fp32", 1e-5)])
def test_ties_vs_oracle_and_energy(prec, ftol, N, levels):
    """N = 2000: one z tile; N = 6000: z buckets with about 100 tied particles
    per z value (both tie orders on the bucket path), or with 500 per value
    (a bucket overflows: tile and merge passes)."""
    cfg = _tied_slab(N=N, levels=levels)
    e = W.engine_for(cfg, prec, mode_flags=L.QEM_EQUAL_Z_TIES)
    k3, sK = e.get_kset()
    F, E = e.forces(cfg["xyz"], cfg["q"], terms=L.QEM_TERM_LONG, energy=True)
    p = O.params(cfg["L"], cfg["alpha"], cfg["r_cutoff"], cfg["gamma_down"], cfg["gamma_up"], z_ties=1)
    Fo = O.F_long(p, cfg["xyz"], cfg["q"], k3, sK)
    assert W.rel_err(F, Fo)[0] <= ftol
    e0 = W.engine_for(cfg, prec)
    F0, E0 = e0.forces(cfg["xyz"], cfg["q"], terms=L.QEM_TERM_LONG, energy=True)
    assert abs(E - E0) <= 1e-12 * abs(E0) if prec == "fp64" else abs(E - E0) <= 1e-6 * abs(E0)
    assert W.rel_err(F0, Fo)[0] > 10 * ftol  # the ties matter here
    # the in-plane components do not depend on the order of ties
    assert np.abs(F[:, :2] - F0[:, :2]).max() <= (1e-12 if prec == "fp64" else 1e-5) * np.abs(F0).max()


def test_ties_flag_is_neutral_without_ties():
    cfg = W.config3(N=3000)
    e = W.engine_for(cfg, "fp64", mode_flags=L.QEM_EQUAL_Z_TIES)
    e0 = W.engine_for(cfg, "fp64")
    F, E = e.forces(cfg["xyz"], cfg["q"], energy=True)
    F0, E0 = e0.forces(cfg["xyz"], cfg["q"], energy=True)
    assert W.rel_err(F, F0)[0] <= 1e-13 and abs(E - E0) <= 1e-13 * abs(E0)


def test_ties_adjoint_vs_fd():
    cfg = _tied_slab(N=400, levels=8, seed=5)
    cfg["P"] = 48
    e = W.engine_for(cfg, "fp64", mode_flags=L.QEM_EQUAL_Z_TIES)
    xyz, q = cfg["xyz"].copy(), cfg["q"].copy()
    rng = np.random.default_rng(2)
    gF = rng.normal(size=xyz.shape)
    gE, h, terms = 0.6, 1e-4, L.QEM_TERM_LONG
    gx, gq, gg = e.backward(xyz, q, gF, gE, terms=terms)
    sx, sq = np.sqrt(np.mean(gx ** 2)), np.sqrt(np.mean(gq ** 2))

    def Lval(x, qq):
        F, E = e.forces(x, qq, terms=terms, energy=True)
        return F, E

    for i in rng.choice(len(q), 5, replace=False):
        for a in (0, 1):  # in-plane moves keep every tie
            xp, xm = xyz.copy(), xyz.copy()
            xp[i, a] += h
            xm[i, a] -= h
            (Fp, Ep), (Fm, Em) = Lval(xp, q), Lval(xm, q)
            fd = (np.sum(gF * (Fp - Fm)) + gE * (Ep - Em)) / (2 * h)
            assert abs(fd - gx[i, a]) <= 2e-6 * (abs(fd) + sx), (i, a, fd, gx[i, a])
        qp, qm = q.copy(), q.copy()
        qp[i] += h
        qm[i] -= h
        (Fp, Ep), (Fm, Em) = Lval(xyz, qp), Lval(xyz, qm)
        fd = (np.sum(gF * (Fp - Fm)) + gE * (Ep - Em)) / (2 * h)
        assert abs(fd - gq[i]) <= 2e-6 * (abs(fd) + sq), (i, fd, gq[i])
    # gamma gradient: both tie orders' parts are summed
    for gi in (0, 1):
        d = dict(gamma_down=cfg["gamma_down"], gamma_up=cfg["gamma_up"])
        key = "gamma_down" if gi == 0 else "gamma_up"
        vals = []
        for sgn in (+1, -1):
            c2 = dict(cfg, **{key: d[key] + sgn * h})
            e2 = W.engine_for(c2, "fp64", mode_flags=L.QEM_EQUAL_Z_TIES)
            e2.set_kset(*e.get_kset())
            vals.append(e2.forces(xyz, q, terms=terms, energy=True))
        fd = (np.sum(gF * (vals[0][0] - vals[1][0])) + gE * (vals[0][1] - vals[1][1])) / (2 * h)
        assert abs(fd - gg[gi]) <= 2e-6 * (abs(fd) + abs(gg).max()), (gi, fd, gg[gi])
