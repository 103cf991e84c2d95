"""gamma_1 gamma_2 > 1 (metamaterial substrates): the regularised short-range
quadrature of python_lib Force_short_norm_njit.py on the GPU (FP64, python
mode) against the reference's own pair and self forces (short_norm.json) and
the oracle on a slab; energies and the short-range adjoint are refused (the
reference defines neither); the long range keeps its plain formulas."""
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
G = float(np.exp(1.0))  # gamma_1 = gamma_2 = e: g12 = e^2, k_0 = 0.5 at Lz = 2


def _engine(Lb, r_c=6.0, alpha=0.1, acc=1e-6, N_t=30, eps=0.05, rbe_p=0):
    return api.Engine(L_box=Lb, alpha=alpha, r_cutoff=r_c, gamma_1=G, gamma_2=G, accuracy=acc, N_t=N_t,
                      rbe_p=rbe_p, mode_flags=L.QEM_PYTHON_MODE, precision=L.QEM_FP64, pv_eps=eps)


def test_pairs_vs_python_norm():
    """Two particles per case: the force on j is the reference's pair force plus its self force."""
    d = json.load(open(os.path.join(GOLD, "short_norm.json")))
    e = _engine((50.0, 50.0, d["L_z"]), r_c=10.0, alpha=d["alpha"], acc=d["accuracy"], N_t=d["N_t"],
                eps=d["pv_eps"])
    for c in d["cases"]:
        xyz = np.array([c["c_i"], c["c_j"]])
        q = np.array([c["q_i"], c["q_j"]])
        F = e.forces(xyz, q, terms=L.QEM_TERM_SHORT)
        ci, cj = np.array(c["c_i"]), np.array(c["c_j"])
        rho = np.hypot(*(cj[:2] - ci[:2]))
        want = np.array([c["F_rho"] * (cj[0] - ci[0]) / rho, c["F_rho"] * (cj[1] - ci[1]) / rho,
                         c["F_z"] + c["F_z_self_j"]])
        np.testing.assert_allclose(F[1], want, rtol=1e-10, atol=1e-13)


def test_slab_vs_oracle_and_refusals():
    rng = np.random.default_rng(21)
    N, Lb = 300, (40.0, 40.0, 2.0)
    xyz = np.stack([Lb[0] * rng.random(N), Lb[1] * rng.random(N), 0.2 + 1.6 * rng.random(N)], 1)
    q = rng.uniform(0.5, 1.5, N) * rng.choice([-1.0, 1.0], N)
    q[-1] -= q.sum()
    e = _engine(Lb)
    F = e.forces(xyz, q, terms=L.QEM_TERM_SHORT)
    p = O.params(Lb, 0.1, 6.0, G, G, accuracy=1e-6, N_t=30, cutoff_mode=O.CUTOFF_PYTHON,
                 dir_mode=O.DIR_MINIMAGE, pair_mode=O.PAIR_PHYSICAL, pv_eps=0.05)
    Fo = O.short_forces(p, xyz, q)
    assert W.rel_err(F, Fo)[0] <= 1e-10
    with pytest.raises(L.QemError):
        e.forces(xyz, q, terms=L.QEM_TERM_SHORT, energy=True)
    with pytest.raises(L.QemError):
        e.backward(xyz, q, np.ones_like(xyz), 0.0, terms=L.QEM_TERM_SHORT)
    # the long range (plain formulas, as in the python_lib) against the oracle
    el = _engine(Lb, rbe_p=40)
    el.sample_kset(3, 40)
    k3, sK = el.get_kset()
    FL = el.forces(xyz, q, terms=L.QEM_TERM_LONG)
    assert W.rel_err(FL, O.F_long(p, xyz, q, k3, sK))[0] <= 1e-9
