"""Pin the FP64 CPU oracle against the reference's own known answers.

Each test restates one assertion of the reference's test-suite (file:line in
the docstring) against golden vectors produced by the reference's numba
python_lib (tests/golden/make_golden.py), at the reference's tolerance, and
where the arithmetic is the same, at a much tighter one.
"""
import json
import os

import numpy as np
import pytest

import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")
SQRT_EPS = np.sqrt(np.finfo(float).eps)  # Julia's default isapprox rtol


def load(name):
    with open(os.path.join(GOLD, name)) as f:
        return json.load(f)


def test_gauss_legendre_exactness():
    """test/Guassian_int.jl:14-48: Step=20 integrates k x^n exactly."""
    rng = np.random.default_rng(1)
    x, w = O.gauss_legendre(20)
    for _ in range(10):
        a, b = np.sort(rng.random(2))
        k, n = rng.integers(1, 6, 2)
        xs = (b + a) / 2 + (b - a) * x / 2
        ws = (b - a) * w / 2
        assert np.isclose(np.sum(ws), b - a, rtol=SQRT_EPS)
        assert np.isclose(np.sum(k * xs ** n * ws), k * (b ** (n + 1) - a ** (n + 1)) / (n + 1), rtol=SQRT_EPS)
    for n in (1, 2, 5, 10, 30, 64):
        xr, wr = np.polynomial.legendre.leggauss(n)
        xo, wo = O.gauss_legendre(n)
        assert np.allclose(xo, xr, atol=1e-15) and np.allclose(wo, wr, rtol=1e-13)


def test_greens_vs_python():
    """test/greens_funtion.jl:7-37 (pair and self Gamma_1/2, dz_Gamma_1/2)."""
    d = load("greens.json")
    assert d["gamma_11111"] == -1.0
    for c in d["cases"]:
        p = O.params((20, 20, c["L_z"]), 1.0, 1.0, c["gamma_1"], c["gamma_2"], accuracy=1e-4)
        e = O.elem_pair(p, c["z_i"], c["z_j"], 1.0)
        es = O.elem_self(p, c["z_i"])
        k = c["k"]
        got = dict(Gamma=O.Gamma_1(p, k, e), Gamma_a=O.Gamma_2(p, k, e), dz_Gamma=O.dz_Gamma_1(p, k, e),
                   dz_Gamma_a=O.dz_Gamma_2(p, k, e), Gamma_self=O.Gamma_1(p, k, es),
                   Gamma_a_self=O.Gamma_2(p, k, es), dz_Gamma_self=O.dz_Gamma_1(p, k, es),
                   dz_Gamma_a_self=O.dz_Gamma_2(p, k, es))
        for name, v in got.items():
            assert np.isclose(v, c[name], rtol=1e-13, atol=1e-300), name


def test_kset_generator_normalised():
    """test/k_gen.jl:3-5: sum(P) == 1 for K_set_generator(1, 1, 0.1, 1e-6)."""
    K, P, sK = O.kset_generator(1, 1, 0.1, 1e-6)
    assert np.isclose(P.astype(np.float64).sum(), 1.0, rtol=SQRT_EPS)
    K, P, sK = O.kset_generator(100.0, 100.0, 0.1, 1e-6)
    assert np.isclose(P.astype(np.float64).sum(), 1.0, rtol=1e-6)
    assert np.all(K[:, 2] > 0)


@pytest.mark.parametrize("fixture", ["short_pair_refbessel.json", "short_pair_accurate.json"])
def test_short_pair_julia_vs_python(fixture):
    """test/Force_short_test.jl:55-93: Julia F_short_ij/F_short_i vs python at atol 1e-5."""
    rho = np.hypot(0.1, 0.2)
    for c in load(fixture)["cases"]:
        p = O.params((10, 10, 2), 0.1, 1.0, c["gamma_1"], c["gamma_2"], accuracy=1e-6, N_t=30)
        F, _ = O.F_short_ij(p, 1, 1, [5.0, 5.0, 0.2], [5.1, 5.2, 0.15])
        Fs = O.F_short_i(p, 1, [5.0, 5.0, 0.2])
        assert np.isclose(F[0], -0.1 / rho * c["F_rs"], atol=1e-5)
        assert np.isclose(F[1], -0.2 / rho * c["F_rs"], atol=1e-5)
        assert np.isclose(F[2], c["F_zs"], atol=1e-5)
        assert np.isclose(Fs[2], c["F_zs_self"], atol=1e-5)


def test_short_pair_python_convention_tight():
    """Same fixture in the python_lib cutoff convention (Force_short_range_njit.py:47-120) with
    accurate Bessel functions: the arithmetic is identical, so agreement is ~1e-15."""
    rho = np.hypot(0.1, 0.2)
    for c in load("short_pair_accurate.json")["cases"]:
        p = O.params((10, 10, 2), 0.1, 1.0, c["gamma_1"], c["gamma_2"], accuracy=1e-9, N_t=30,
                     cutoff_mode=O.CUTOFF_PYTHON)
        F, _ = O.F_short_ij(p, 1, 1, [5.0, 5.0, 0.2], [5.1, 5.2, 0.15])
        Fs = O.F_short_i(p, 1, [5.0, 5.0, 0.2])
        ref = np.array([-0.1 / rho * c["F_rs"], -0.2 / rho * c["F_rs"], c["F_zs"]])
        assert np.allclose(F, ref, rtol=1e-12, atol=0)
        assert np.isclose(Fs[2], c["F_zs_self"], rtol=1e-12)


def test_short_pair_vs_icm():
    """test/Force_short_test.jl:9-45: point-charge part (single=true) vs ICM image sum, atol 1e-5."""
    for c in load("short_pair_refbessel.json")["cases"]:
        p = O.params((10, 10, 2), 1.0, 1.0, c["gamma_1"], c["gamma_2"], accuracy=1e-6, N_t=30)
        F, _ = O.F_short_ij(p, 1, 1, [5.0, 5.0, 0.2], [5.1, 5.2, 0.15], single=True)
        Fs = O.F_short_i(p, 1, [5.0, 5.0, 0.2], single=True)
        assert np.allclose(F, [c["icm_Fx"], c["icm_Fy"], c["icm_Fz"]], atol=1e-5)
        assert np.isclose(Fs[2], c["icm_Fzs"], atol=1e-5)


def test_icm_three_particles():
    """ICM.py:71-123 (image-charge force) vs the sum of single=true pair and self forces."""
    d = load("icm_energy.json")
    P = np.array(d["POSCAR"])
    xyz, q = P[:, 1:], P[:, 0]
    p = O.params(d["L"], 1.0, 1.0e5, d["gamma_1"], d["gamma_2"], accuracy=1e-10, N_t=60)
    F = np.zeros((3, 3))
    for i in range(3):
        for j in range(3):
            if i != j:
                F[i] += O.F_short_ij(p, q[i], q[j], xyz[i], xyz[j], single=True)[0]
        F[i] += O.F_short_i(p, q[i], xyz[i], single=True)
    icm = np.array(d["F"])  # Fx, Fy, Fz, Fxs, Fys, Fzs rows
    ref = np.stack([icm[0], icm[1], icm[2] + icm[5]], 1)
    assert np.allclose(F, ref, atol=1e-6)


def test_long_range_four_particles():
    """test/Force_long_test.jl:1-293: Fl_non_sort, Fl_sort (z sign flip at 108), Flz_sort_k0,
    Flz_self and F_l_total against Sigma_Gamma_func_njit, z_list = [2, 1, 3, 4]."""
    d = load("long_4particle.json")
    P4 = np.array(d["POSCAR"])
    xyz, q = P4[:, 1:], P4[:, 0]
    zl = np.array([1, 0, 2, 3])
    for c in d["cases"]:
        k3 = np.array([c["kx"], c["ky"], np.hypot(c["kx"], c["ky"])])
        g1, g2 = c["gamma_1"], c["gamma_2"]
        s1 = np.array(c["sum1"]).T
        s2 = np.array(c["xy_sum2"]).T
        z2 = np.array(c["z_sum2"])
        assert np.allclose(O.Fl_non_sort(k3, xyz, q, g1, g2, 2.0), s1, rtol=1e-13, atol=1e-15)
        b = O.Fl_sort(k3, zl, xyz, q)
        assert np.allclose(b[:, :2], s2, rtol=1e-13, atol=1e-15)
        assert np.allclose(-b[:, 2], z2, rtol=1e-13, atol=1e-15)
        assert np.allclose(O.Flz_sort_k0(zl, q)[:, 2], c["z_sum0"], rtol=1e-15, atol=1e-15)
        assert np.allclose(O.Flz_self(k3, xyz, q, g1, g2, 2.0)[:, 2], c["z_self"], rtol=1e-13)
        p = O.params((10, 10, 2), 1.0, 1.0, g1, g2)
        t = O.F_l_total(p, k3, xyz, q, zl)
        Fpy = np.stack([(s1[:, 0] + s2[:, 0]) / 100, (s1[:, 1] + s2[:, 1]) / 100,
                        (s1[:, 2] - z2 + np.array(c["z_self"])) / 100], 1)
        assert np.allclose(t, Fpy, rtol=1e-12, atol=1e-15)
        assert np.isclose(O.sigma_s(k3, xyz, q, g1, g2, 2.0), c["sigma_s"], rtol=1e-13)
        assert np.isclose(O.sigma_ns(k3, xyz, q, zl), c["sigma_ns"], rtol=1e-13)


def test_system_python_convention():
    """60-particle slab through the python_lib drivers: pair set, short forces, energies and the
    random-batch long range assembled for a fixed k-set (system_python.json)."""
    d = load("system_python.json")
    xyz, q = np.array(d["xyz"]), np.array(d["q"])
    p = O.params(d["L"], d["alpha"], d["r_cutoff"], d["gamma_1"], d["gamma_2"], accuracy=d["accuracy"],
                 N_t=d["N_t"], cutoff_mode=O.CUTOFF_PYTHON, dir_mode=O.DIR_MINIMAGE, pair_mode=O.PAIR_PHYSICAL)
    pl = O.pairs(p, xyz)
    ref_pairs = {(min(i, j), max(i, j)) for j, r in enumerate(d["pairs_full"]) for i in r}
    assert set(map(tuple, pl.tolist())) == ref_pairs
    assert set(map(tuple, O.pairs(p, xyz, method="cells").tolist())) == ref_pairs
    F = O.short_forces(p, xyz, q, pl)
    Fr = np.array(d["F_short"])
    assert np.abs(F - Fr).max() <= 1e-12 * np.abs(Fr).max()
    assert np.isclose(O.energy_short(p, xyz, q, pl), d["E_short"], rtol=1e-12)
    ks = np.array(d["kset"])
    k3 = np.concatenate([ks, np.hypot(ks[:, 0], ks[:, 1])[:, None]], 1)
    FL = O.F_long(p, xyz, q, k3, d["sum_K"])
    assert np.abs(FL - np.array(d["F_long"])).max() <= 1e-12 * np.abs(FL).max()
    assert np.isclose(O.energy_long(p, xyz, q, k3, d["sum_K"]), d["E_long_k"] + d["E_long_k0"], rtol=1e-12)


def test_exact_long_range_vs_python_exact():
    """Exact k-sum (every lattice vector 0 < k < k_c, weights e^{-k^2/4 alpha}) against
    Force_long_range_njit_exact.Force_long_cal (long_exact.json)."""
    d = load("long_exact.json")
    xyz, q = np.array(d["xyz"]), np.array(d["q"])
    p = O.params(d["L"], d["alpha"], 1.0, d["gamma_1"], d["gamma_2"])
    k3, w = O.exact_kset(d["L"], d["alpha"], d["k_cutoff"])
    assert k3.shape[0] == d["n_k"]
    assert np.all((k3[:, 2] > 0) & (k3[:, 2] < d["k_cutoff"]))
    np.testing.assert_allclose(k3[:, 2], np.hypot(k3[:, 0], k3[:, 1]), rtol=1e-15)
    np.testing.assert_allclose(w, np.exp(-k3[:, 2] ** 2 / (4 * d["alpha"])), rtol=1e-15)
    F = O.F_long_weighted(p, xyz, q, k3, w)
    Fr = np.array(d["F_long"])
    assert np.abs(F - Fr).max() <= 1e-12 * np.abs(Fr).max()
    # the weighted form with uniform weights is the random-batch F_long
    rng = np.random.default_rng(3)
    sel = rng.choice(k3.shape[0], 9, replace=False)
    np.testing.assert_allclose(O.F_long_weighted(p, xyz, q, k3[sel], np.full(9, 2.5 / 9)),
                               O.F_long(p, xyz, q, k3[sel], 2.5), rtol=0, atol=1e-15 * np.abs(Fr).max())
    assert np.isclose(O.energy_long_weighted(p, xyz, q, k3[sel], np.full(9, 2.5 / 9)),
                      O.energy_long(p, xyz, q, k3[sel], 2.5), rtol=1e-14)


def test_equal_z_ties_vs_python_equal_cell():
    """Particles on 5 z levels (long_ties.json): with z_ties the oracle's z-ordered sums count
    equal-z particles as neither below nor above (python_lib equal_cell); the plain sortperm
    order differs in F_z only, and the k = 0 energy does not depend on it."""
    d = load("long_ties.json")
    xyz, q = np.array(d["xyz"]), np.array(d["q"])
    ks = np.array(d["kset"])
    k3 = np.concatenate([ks, np.hypot(ks[:, 0], ks[:, 1])[:, None]], 1)
    Fr = np.array(d["F_long"])
    zl = np.argsort(xyz[:, 2], kind="stable").astype(np.int32)
    p = O.params(d["L"], 1.0, 1.0, d["gamma_1"], d["gamma_2"], z_ties=1)
    F = O.F_long(p, xyz, q, k3, d["sum_K"])
    assert np.abs(F - Fr).max() <= 1e-12 * np.abs(Fr).max()
    assert np.isclose(O.energy_k0(p, xyz, q, zl), d["E_long_k0"], rtol=1e-13)
    p0 = O.params(d["L"], 1.0, 1.0, d["gamma_1"], d["gamma_2"])
    F0 = O.F_long(p0, xyz, q, k3, d["sum_K"])
    assert np.abs(F0[:, :2] - Fr[:, :2]).max() <= 1e-12 * np.abs(Fr).max()
    assert np.abs(F0[:, 2] - Fr[:, 2]).max() > 0.05 * np.abs(Fr).max()


def test_regularised_quadrature_vs_python_norm():
    """gamma_1 gamma_2 > 1 (short_norm.json): the oracle's pair and self forces in python
    mode against Force_rhos_norm / Force_zs_norm / Force_zs_self_norm."""
    import ctypes as C

    d = load("short_norm.json")
    p = O.params((50.0, 50.0, d["L_z"]), d["alpha"], 10.0, d["gamma_1"], d["gamma_2"], accuracy=d["accuracy"],
                 N_t=d["N_t"], cutoff_mode=O.CUTOFF_PYTHON, dir_mode=O.DIR_MINIMAGE, pair_mode=O.PAIR_PHYSICAL,
                 pv_eps=d["pv_eps"])
    L = O.lib()
    for c in d["cases"]:
        cj, ci = np.array(c["c_j"]), np.array(c["c_i"])
        out = np.zeros(4)
        L.qo_F_short_ij(C.byref(p), c["q_j"], c["q_i"], O._d(cj)[1], O._d(ci)[1], 0, O._d(out)[1])
        rho = np.hypot(cj[0] - ci[0], cj[1] - ci[1])
        assert np.isclose(out[0], c["F_rho"] * (cj[0] - ci[0]) / rho, rtol=1e-12, atol=0)
        assert np.isclose(out[1], c["F_rho"] * (cj[1] - ci[1]) / rho, rtol=1e-12, atol=0)
        assert np.isclose(out[2], c["F_z"], rtol=1e-11, atol=0)
        assert np.isclose(L.qo_F_short_i(C.byref(p), c["q_j"], O._d(cj)[1], 0), c["F_z_self_j"], rtol=1e-12)


def test_sortperm_is_stable():
    """QEM_long.jl:39-40 sortperm: stable ascending, ties keep index order."""
    rng = np.random.default_rng(3)
    z = np.round(rng.random(500) * 20) / 2  # many ties
    xyz = np.stack([np.zeros(500), np.zeros(500), z], 1)
    assert np.array_equal(O.sortperm_z(xyz), np.argsort(z, kind="stable"))


def test_lj_wall_semantics():
    """Substrate_LJ.jl:34-43: F_z = dir*24 eps/dz^2 (2 s^12 - s^6) when dz < cutoff (signed dz)."""
    xyz = np.array([[0, 0, 0.5], [0, 0, 3.0], [0, 0, 9.7]])
    F, bad = O.lj_forces(xyz, 1.0, 1.0, 1.0, 0.0, +1)
    dz = 0.5
    s6 = (1 / dz ** 2) ** 3
    assert bad == 0 and np.isclose(F[0, 2], 24 / dz ** 2 * (2 * s6 * s6 - s6)) and F[1, 2] == 0 and F[2, 2] == 0
    F, bad = O.lj_forces(xyz, 1.0, 1.0, 1.0, 10.0, -1)
    assert bad == 0 and np.all(F[:, 2] != 0)  # signed dz < cutoff holds for every particle
    F, bad = O.lj_forces(np.array([[0, 0, -0.1]]), 1.0, 1.0, 1.0, 0.0, +1)
    assert bad == 1
