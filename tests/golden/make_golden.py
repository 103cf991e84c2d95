"""Generate golden vectors for the QEM oracle from the reference's own code.

Run where a checkout of the reference (ArrogantGao/QEM4Molly) exists; its
root is taken from ``--reference DIR`` or the ``QEM_REFERENCE_DIR``
environment variable, and defaults to ``/root/reference``.  The fixtures it
writes (``tests/golden/*.json``) are committed, so the test-suite and the GPU
box never need the reference tree.

    python tests/golden/make_golden.py [--reference DIR]   # writes all fixtures

What is generated (each case states the reference file it exercises):

* ``greens.json``      -- test/greens_funtion.jl:10-37: 100 random cases of
  green_norm_njit.Gamma / Gamma_a / dz_Gamma / dz_Gamma_a (pair and self).
* ``short_pair.json``  -- test/Force_short_test.jl: the 2-particle fixture,
  ICM.F_cal with 100 image layers (lines 9-45) and
  Force_short_range_njit.Force_rhos_ji / Force_zs_ji / Force_zs_self_ji
  (lines 55-93), for 10 seeded (gamma_1, gamma_2) draws; once with the
  reference's own Bessel module and once with an accurate-Bessel shim.
* ``long_4particle.json`` -- test/Force_long_test.jl: the 4-particle fixture
  with z_list [2, 1, 3, 4]; Sigma_Gamma_func_njit.F_long_sum_1,
  F_long_xy_sum_2, F_long_z_sum_2 and F_long_z_self_sum for seeded k and
  gamma draws.
* ``system_python.json`` -- a 60-particle slab evaluated by the python_lib
  drivers (Force_short_cal + neighbor_check, the long-range sums assembled as
  Force_long_range_njit.Force_long_cal does for a fixed k-set,
  Energy_short_cal, Sigma_Gamma_func_s/_ns and Energy_long_kzero) with the
  accurate-Bessel shim, so the python-convention oracle mode is pinned to
  ~1e-12.
* ``icm_energy.json``  -- ICM.U_cal / ICM.F_cal on a 3-particle slab.
* ``short_norm.json``  -- gamma_1 gamma_2 > 1: the regularised pair and self
  forces of Force_short_norm_njit.py for 12 seeded pairs (accurate Bessel).
* ``long_ties.json``   -- equal-z ties: a 36-particle slab on 5 z levels
  through the z-ordered sums with their equal_cell groups (fixed k-set).
* ``long_exact.json``  -- the exact (non-random-batch) long range of
  Force_long_range_njit_exact.Force_long_cal on a 24-particle slab, with every
  lattice vector up to the cutoff (k-sorted rows, so its k <= k_f1 loop takes
  exactly that set).

The accurate-Bessel shim replaces the python_lib ``Bessel`` module (whose J1
has ~1.5e-5 absolute error) by numba functions calling libm's j0/j1, exactly
the functions the oracle uses.  Each variant runs in its own subprocess because
numba binds module globals at compile time.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile
import types

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_REFERENCE = "/root/reference"


def _reference_root(argv):
    for i, a in enumerate(argv):
        if a.startswith("--reference="):
            return a.split("=", 1)[1]
        if a == "--reference" and i + 1 < len(argv):
            return argv[i + 1]
    return os.environ.get("QEM_REFERENCE_DIR", DEFAULT_REFERENCE)


REF_LIB = os.path.join(_reference_root(sys.argv[1:]), "src", "python_lib")


def _setup(bessel: str):
    os.environ.setdefault("NUMBA_CACHE_DIR", tempfile.mkdtemp(prefix="numba_cache_"))
    sys.dont_write_bytecode = True
    # ICM.py imports matplotlib.pyplot at module level; it is never used.
    mpl = types.ModuleType("matplotlib")
    mpl.pyplot = types.ModuleType("matplotlib.pyplot")
    sys.modules.setdefault("matplotlib", mpl)
    sys.modules.setdefault("matplotlib.pyplot", mpl.pyplot)
    if bessel == "accurate":
        import ctypes

        import numba

        libm = ctypes.CDLL("libm.so.6")
        _j0 = libm.j0
        _j0.restype = ctypes.c_double
        _j0.argtypes = [ctypes.c_double]
        _j1 = libm.j1
        _j1.restype = ctypes.c_double
        _j1.argtypes = [ctypes.c_double]

        @numba.njit
        def Bessel0(x):
            return _j0(x)

        @numba.njit
        def Bessel1(x):
            return _j1(x)

        shim = types.ModuleType("Bessel")
        shim.Bessel0 = Bessel0
        shim.Bessel1 = Bessel1
        sys.modules["Bessel"] = shim
    sys.path.insert(0, REF_LIB)


def gen_greens(rng):
    import green_norm_njit as g

    cases = []
    for _ in range(100):
        k, e1, e2, e3, _lz = rng.random(5)
        Lz = 10.0
        zi, zj = 10.0 * rng.random(2)
        cases.append(dict(
            k=k, eps_1=e1, eps_2=e2, eps_3=e3, L_z=Lz, z_i=zi, z_j=zj,
            gamma_1=(e2 - e1) / (e2 + e1), gamma_2=(e2 - e3) / (e2 + e3),
            Gamma=g.Gamma(k, e1, e2, e3, Lz, zj, zi),
            Gamma_a=g.Gamma_a(k, e1, e2, e3, Lz, zj, zi),
            dz_Gamma=g.dz_Gamma(k, e1, e2, e3, Lz, zi, zj),
            dz_Gamma_a=g.dz_Gamma_a(k, e1, e2, e3, Lz, zi, zj),
            Gamma_self=g.Gamma(k, e1, e2, e3, Lz, zi, zi),
            Gamma_a_self=g.Gamma_a(k, e1, e2, e3, Lz, zi, zi),
            dz_Gamma_self=g.dz_Gamma_self(k, e1, e2, e3, Lz, zi, zi),
            dz_Gamma_a_self=g.dz_Gamma_a_self(k, e1, e2, e3, Lz, zi, zi),
        ))
    return dict(source="test/greens_funtion.jl:10-37 via green_norm_njit.py:6-168",
                gamma_11111=g.gamma(1, 1, 1, 1, 1), cases=cases)


def gen_short_pair(rng, bessel):
    import numpy as np

    import Force_short_range_njit as Fs
    import ICM

    out = []
    for _ in range(10):
        g1, g2 = rng.random(2)
        e1 = (1 - g1) / (1 + g1)
        e3 = (1 - g2) / (1 + g2)
        INCAR = np.array([2, 1e-9, 10, 10, 2, e1, 1, e3, 0.1, 1e-9], dtype=float)
        POSCAR = np.array([[1, 5.0, 5.0, 0.2], [1, 5.1, 5.2, 0.15]], dtype=float)
        N_image = 100
        POS = np.zeros([2 * N_image + 1, 2, 4])
        icm = ICM.F_cal(INCAR, POSCAR, POS, N_image, 0) if bessel == "ref" else None
        G1 = np.polynomial.legendre.leggauss(30)
        G2 = np.polynomial.legendre.leggauss(30)
        pos_info = np.array([1, 1, 5.0, 5.1, 5.0, 5.2, 0.2, 0.15])
        F_rs = Fs.Force_rhos_ji(pos_info, INCAR, G1, G2, 1)
        F_zs = Fs.Force_zs_ji(pos_info, INCAR, G1, G2, 1)
        F_zs_self = Fs.Force_zs_self_ji(np.array([1, 5.0, 5.0, 0.2]), INCAR, G1, G2, 1)
        case = dict(gamma_1=g1, gamma_2=g2, F_rs=F_rs, F_zs=F_zs, F_zs_self=F_zs_self)
        if icm is not None:
            case.update(icm_Fx=icm[0][0], icm_Fy=icm[1][0], icm_Fz=icm[2][0], icm_Fzs=icm[5][0])
        out.append(case)
    return out


def gen_long_4(rng):
    import numpy as np

    import Sigma_Gamma_func_njit as S

    POSCAR = np.array([[1, 5.0, 5.0, 0.2], [-1, 5.1, 5.2, 0.15], [1, 4.9, 4.9, 0.3], [-1, 5.5, 5.3, 0.4]])
    Lz = 2.0
    zl = np.array([1, 0, 2, 3])
    eq_cell = np.array([[1], [0], [2], [3]])
    eq_size = np.array([1, 2, 3, 4])
    cases = []
    for t in range(10):
        if t == 0:
            kx, ky = 1.0, 1.0  # test/Force_long_test.jl:16-17
        else:
            kx, ky = rng.random(2)
        g1, g2 = rng.random(2)
        K = kx * kx + ky * ky
        k = np.sqrt(K)
        kset = np.array([kx, ky, K, k])
        e1 = (1 - g1) / (1 + g1)
        e3 = (1 - g2) / (1 + g2)
        s1 = S.F_long_sum_1(kset, e1, 1, e3, POSCAR, Lz)
        s2 = S.F_long_xy_sum_2(kset, POSCAR, zl)
        z0, z2 = S.F_long_z_sum_2(kset, POSCAR, zl, eq_cell, eq_size, 4)
        zs = S.F_long_z_self_sum(kset, POSCAR, e1, 1, e3, Lz)
        cases.append(dict(kx=kx, ky=ky, gamma_1=g1, gamma_2=g2,
                          sum1=[list(a) for a in s1], xy_sum2=[list(a) for a in s2],
                          z_sum0=list(z0), z_sum2=list(z2), z_self=list(zs),
                          sigma_s=S.Sigma_Gamma_func_s(kset, e1, 1, e3, POSCAR, Lz),
                          sigma_ns=S.Sigma_Gamma_func_ns(kset, POSCAR, zl)))
    return dict(source="test/Force_long_test.jl:13-37 via Sigma_Gamma_func_njit.py:8-304",
                POSCAR=POSCAR.tolist(), L=[10.0, 10.0, 2.0], z_list_py=zl.tolist(), cases=cases)


def gen_system(rng):
    import numpy as np

    import cell_list
    import Energy_long_range_njit as El
    import Energy_short_range_njit as Es
    import Force_short_range_njit as Fs
    import neighbor_check
    import Sigma_Gamma_func_njit as S

    N, Lx, Ly, Lz = 60, 30.0, 30.0, 5.0
    alpha, r_c, acc, N_t = 0.1, 6.0, 1e-6, 30
    g1, g2 = -0.6, 0.8  # gamma_down, gamma_up
    e1 = (1 - g1) / (1 + g1)
    e3 = (1 - g2) / (1 + g2)
    q = np.array([1.0 if i % 2 == 0 else -1.0 for i in range(N)])
    x = rng.random(N) * Lx
    y = rng.random(N) * Ly
    z = 0.5 + rng.random(N) * (Lz - 1.0)
    POSCAR = np.stack([q, x, y, z], axis=1)
    nc = int(Lx // r_c)
    INCAR = dict(NUM_particle=N, L_x=Lx, L_y=Ly, L_z=Lz, alpha=alpha, r_c=r_c,
                 Cell_info=(nc, nc, 1, Lx / nc, Ly / nc, Lz))
    CELL = cell_list.Cell_create(POSCAR, INCAR)
    rows = []
    for j in range(N):
        nb = neighbor_check.neighbor_check(j, POSCAR, INCAR, CELL)
        rows.append([[m[0], m[1], m[2], m[3], np.sqrt((x[j] - m[1]) ** 2 + (y[j] - m[2]) ** 2), m[4]] for m in nb])
    M = max(len(r) for r in rows)
    nbl = np.full([N, M + 1, 5], 9999.0)
    for j, r in enumerate(rows):
        for t, m in enumerate(r):
            nbl[j, t] = m[:5]
    k_f1 = np.sqrt(-4 * alpha * np.log(acc))
    k_f2 = -np.log(acc) / (2 * Lz)
    G = np.polynomial.legendre.leggauss(N_t)
    gg = Fs.Gauss_para_gen(-1.1, 1, -1.1, Lz, 50, acc, alpha)
    Fx, Fy, Fz = Fs.Force_short_cal(nbl, 1.0, e1, 1.0, e3, Lz, alpha, POSCAR, G, G, k_f1, k_f2, N_t, acc,
                                   0.0, *gg)
    Gt = np.array(G).T.copy()
    E_short = Es.Energy_short_cal(nbl, 1.0, e1, 1.0, e3, Lz, alpha, POSCAR, Gt, Gt, k_f1, k_f2)
    # long range: Force_long_range_njit.Force_long_cal's assembly with a fixed k-set
    zl = np.argsort(z, kind="stable")
    eq_cell = zl.reshape(N, 1).copy()
    eq_size = np.arange(1, N + 1)
    P = 12
    mx = rng.integers(-4, 5, P)
    my = rng.integers(-4, 5, P)
    for t in range(P):
        if mx[t] == 0 and my[t] == 0:
            mx[t] = 1
    kset = np.stack([2 * np.pi * mx / Lx, 2 * np.pi * my / Ly], axis=1)
    S_tot = 3.7  # any positive normaliser: it only scales the k != 0 sum
    FLx = np.zeros(N)
    FLy = np.zeros(N)
    FLz = np.zeros(N)
    Es_k = 0.0
    Ens_k = 0.0
    for t in range(P):
        kx, ky = kset[t]
        K = kx * kx + ky * ky
        k4 = np.array([kx, ky, K, np.sqrt(K)])
        a1 = S.F_long_sum_1(k4, e1, 1.0, e3, POSCAR, Lz)
        a2 = S.F_long_xy_sum_2(k4, POSCAR, zl)
        z0, z2 = S.F_long_z_sum_2(k4, POSCAR, zl, eq_cell, eq_size, N)
        zs = S.F_long_z_self_sum(k4, POSCAR, e1, 1.0, e3, Lz)
        w = (1 / (Lx * Ly)) * (S_tot / P)
        FLx += w * (a1[0] + a2[0])
        FLy += w * (a1[1] + a2[1])
        FLz += w * (a1[2] - z2 + zs)
        Es_k += -(S_tot / P) * S.Sigma_Gamma_func_s(k4, e1, 1.0, e3, POSCAR, Lz) / (2 * Lx * Ly)
        Ens_k += -(S_tot / P) * S.Sigma_Gamma_func_ns(k4, POSCAR, zl) / (2 * Lx * Ly)
    FLz += (1 / (2 * Lx * Ly)) * z0
    E_k0 = El.Energy_long_kzero(POSCAR, P, P, kset, Lx, Ly, Lz, 1.0, e1, 1.0, e3, S_tot, zl, eq_cell, eq_size, N)
    return dict(
        source="Force_short_range_njit.py:233-256, Energy_short_range_njit.py:84-99, "
               "Force_long_range_njit.py:16-38 (fixed k-set), Energy_long_range_njit.py:10-44",
        N=N, L=[Lx, Ly, Lz], alpha=alpha, r_cutoff=r_c, accuracy=acc, N_t=N_t, gamma_1=g1, gamma_2=g2,
        q=q.tolist(), xyz=np.stack([x, y, z], 1).tolist(),
        pairs_full=[[int(m[5]) for m in r] for r in rows],
        F_short=np.stack([Fx, Fy, Fz], 1).tolist(), E_short=E_short,
        kset=kset.tolist(), sum_K=S_tot, F_long=np.stack([FLx, FLy, FLz], 1).tolist(),
        E_long_k=Es_k + Ens_k, E_long_k0=E_k0)


def gen_exact(rng):
    """Exact (non-random-batch) long range: Force_long_range_njit_exact.Force_long_cal on a
    24-particle slab.  Its loop takes KCAR rows while k <= k_f1 (line 19); the rows given
    here are every lattice vector sorted by k, with one row past the cutoff, so the sum runs
    over exactly {0 < k <= k_f1}, each k weighted by e^{-k^2/4 alpha} (lines 29-34)."""
    import numpy as np

    import Force_long_range_njit_exact as FE

    N, Lx, Ly, Lz = 24, 12.0, 10.0, 3.0
    alpha, k_c = 0.8, 2.95
    g1, g2 = 0.6, -0.45  # gamma_down, gamma_up
    e1 = (1 - g1) / (1 + g1)
    e3 = (1 - g2) / (1 + g2)
    q = np.array([1.0 if i % 2 == 0 else -1.0 for i in range(N)])
    x = rng.random(N) * Lx
    y = rng.random(N) * Ly
    z = 0.3 + rng.random(N) * (Lz - 0.6)
    POSCAR = np.stack([q, x, y, z], axis=1)
    M = int(k_c * max(Lx, Ly) / (2 * np.pi)) + 2
    rows = []
    for m1 in range(-M, M + 1):
        for m2 in range(-M, M + 1):
            if m1 == 0 and m2 == 0:
                continue
            kx, ky = 2 * np.pi * m1 / Lx, 2 * np.pi * m2 / Ly
            K = kx * kx + ky * ky
            rows.append([kx, ky, K, np.sqrt(K)])
    rows.sort(key=lambda r: r[3])
    KCAR = np.array(rows)
    n_in = int(np.sum(KCAR[:, 3] <= k_c))
    assert np.min(np.abs(KCAR[:, 3] - k_c)) > 1e-9 and n_in < len(rows)
    KCAR = KCAR[: n_in + 1].copy()
    zl = np.argsort(z, kind="stable")
    eq_cell = zl.reshape(N, 1).copy()
    eq_size = np.arange(1, N + 1)
    Fx, Fy, Fz, Fzs = FE.Force_long_cal(POSCAR, KCAR, k_c, alpha, Lx, Ly, Lz, 1.0, e1, 1.0, e3, 0.0, zl, eq_cell,
                                        eq_size, N)
    return dict(source="Force_long_range_njit_exact.py:10-45 (Force_long_cal), z force plus its self part",
                N=N, L=[Lx, Ly, Lz], alpha=alpha, k_cutoff=k_c, gamma_1=g1, gamma_2=g2, n_k=n_in,
                q=q.tolist(), xyz=np.stack([x, y, z], 1).tolist(),
                F_long=np.stack([Fx, Fy, Fz + Fzs], 1).tolist())


def gen_ties(rng):
    """Equal-z ties: a 36-particle slab on 5 z levels through the python_lib z-ordered sums
    with their equal_cell groups (Sigma_Gamma_func_njit.F_long_z_sum_2), assembled for a fixed
    k-set as Force_long_range_njit.Force_long_cal does; also the k = 0 energy."""
    import numpy as np

    import Energy_long_range_njit as El
    import Sigma_Gamma_func_njit as S

    N, Lx, Ly, Lz = 36, 18.0, 15.0, 4.0
    g1, g2 = -0.5, 0.7  # gamma_down, gamma_up
    e1 = (1 - g1) / (1 + g1)
    e3 = (1 - g2) / (1 + g2)
    q = rng.uniform(0.5, 1.5, N) * np.where(np.arange(N) % 2 == 0, 1.0, -1.0)
    q[-1] -= q.sum()
    x = rng.random(N) * Lx
    y = rng.random(N) * Ly
    z = rng.choice(np.array([0.5, 1.25, 2.0, 2.75, 3.5]), N)
    POSCAR = np.stack([q, x, y, z], axis=1)
    zl = np.argsort(z, kind="stable")
    levels = [zl[z[zl] == v] for v in np.unique(z)]
    G = len(levels)
    eq_cell = np.full([G, max(len(m) for m in levels)], 9999)
    for g, m in enumerate(levels):
        eq_cell[g, :len(m)] = m
    eq_size = np.cumsum([len(m) for m in levels])
    P = 10
    mx = rng.integers(-3, 4, P)
    my = rng.integers(-3, 4, P)
    for t in range(P):
        if mx[t] == 0 and my[t] == 0:
            my[t] = 2
    kset = np.stack([2 * np.pi * mx / Lx, 2 * np.pi * my / Ly], axis=1)
    S_tot = 2.3
    FL = np.zeros((N, 3))
    for t in range(P):
        kx, ky = kset[t]
        K = kx * kx + ky * ky
        k4 = np.array([kx, ky, K, np.sqrt(K)])
        a1 = S.F_long_sum_1(k4, e1, 1.0, e3, POSCAR, Lz)
        a2 = S.F_long_xy_sum_2(k4, POSCAR, zl)
        z0, z2 = S.F_long_z_sum_2(k4, POSCAR, zl, eq_cell, eq_size, G)
        zs = S.F_long_z_self_sum(k4, POSCAR, e1, 1.0, e3, Lz)
        w = (1 / (Lx * Ly)) * (S_tot / P)
        FL[:, 0] += w * (a1[0] + a2[0])
        FL[:, 1] += w * (a1[1] + a2[1])
        FL[:, 2] += w * (a1[2] - z2 + zs)
    FL[:, 2] += (1 / (2 * Lx * Ly)) * z0
    E_k0 = El.Energy_long_kzero(POSCAR, P, P, kset, Lx, Ly, Lz, 1.0, e1, 1.0, e3, S_tot, zl, eq_cell, eq_size, G)
    return dict(source="Sigma_Gamma_func_njit.py:8-304 with equal_cell groups, Energy_long_range_njit.py:25-44",
                N=N, L=[Lx, Ly, Lz], gamma_1=g1, gamma_2=g2, q=q.tolist(), xyz=np.stack([x, y, z], 1).tolist(),
                kset=kset.tolist(), sum_K=S_tot, F_long=FL.tolist(), E_long_k0=E_k0, n_levels=G)


def gen_norm(rng):
    """gamma_1 gamma_2 > 1 (metamaterial substrates): the regularised short-range quadrature of
    Force_short_norm_njit.py (Force_rhos_norm, Force_zs_norm, Force_zs_self_norm) with the node
    sets of Force_short_range_njit.Gauss_para_gen, for seeded pairs and particles."""
    import numpy as np

    import Force_short_norm_njit as FN
    import Force_short_range_njit as Fs

    Lz, alpha, acc, N_t, eps = 2.0, 0.1, 1e-6, 30, 0.05
    g1 = g2 = float(np.e)  # gamma_down = gamma_up: g12 = e^2, k_0 = 0.5
    e1 = (1 - g1) / (1 + g1)
    e3 = (1 - g2) / (1 + g2)
    G = Fs.Gauss_para_gen(e1, 1.0, e3, Lz, N_t, acc, alpha)
    INCAR = (1, 1, 1, 1, Lz, e1, 1.0, e3, alpha, acc)
    cases = []
    for t in range(12):
        zi, zj = 0.2 + 1.6 * rng.random(2)
        rho = 0.3 + 2.7 * rng.random()
        ang = 2 * np.pi * rng.random()
        xi, yi = 5.0, 5.0
        xj, yj = xi + rho * np.cos(ang), yi + rho * np.sin(ang)
        qi, qj = (1.0, -1.0) if t % 2 == 0 else (0.7, 1.3)
        pos = (qj, qi, xj, xi, yj, yi, zj, zi)
        cases.append(dict(q_i=qi, q_j=qj, c_i=[xi, yi, zi], c_j=[xj, yj, zj],
                          F_rho=FN.Force_rhos_norm(pos, INCAR, eps, N_t, *G),
                          F_z=FN.Force_zs_norm(pos, INCAR, eps, N_t, *G),
                          F_z_self_j=FN.Force_zs_self_norm((qj, xj, yj, zj), INCAR, eps, N_t, *G)))
    return dict(source="Force_short_norm_njit.py:68-414 with Force_short_range_njit.Gauss_para_gen (258-286)",
                L_z=Lz, alpha=alpha, accuracy=acc, N_t=N_t, pv_eps=eps, gamma_1=g1, gamma_2=g2, cases=cases)


def gen_icm(rng):
    import numpy as np

    import ICM

    g1, g2 = -0.5, 0.7
    e1 = (1 - g1) / (1 + g1)
    e3 = (1 - g2) / (1 + g2)
    Lx = Ly = 1.0e6  # no in-plane periodic images matter (N_real = 0)
    Lz = 3.0
    POSCAR = np.array([[1.0, 1.0, 1.0, 0.7], [-1.0, 1.6, 0.8, 1.9], [1.0, 0.5, 1.9, 2.4]])
    INCAR = np.array([3, 1e-9, Lx, Ly, Lz, e1, 1.0, e3, 0.1, 1e-9])
    N_image = 200
    F = ICM.F_cal(INCAR, POSCAR, np.zeros([2 * N_image + 1, 3, 4]), N_image, 0)
    U = ICM.U_cal(INCAR, POSCAR, np.zeros([2 * N_image + 1, 3, 4]), N_image, 0)
    return dict(source="ICM.py:71-168", gamma_1=g1, gamma_2=g2, L=[Lx, Ly, Lz], N_image=N_image,
                POSCAR=POSCAR.tolist(), F=[list(a) for a in F], U=U)


def _tolist(o):
    import numpy as np

    if isinstance(o, dict):
        return {k: _tolist(v) for k, v in o.items()}
    if isinstance(o, (list, tuple)):
        return [_tolist(v) for v in o]
    if isinstance(o, np.ndarray):
        return _tolist(o.tolist())
    if isinstance(o, (np.floating,)):
        return float(o)
    if isinstance(o, (np.integer,)):
        return int(o)
    return o


def _dump(name, obj):
    import numba
    import numpy as np

    obj = _tolist(obj)
    obj["generator"] = dict(script="tests/golden/make_golden.py", numpy=np.__version__, numba=numba.__version__)
    with open(os.path.join(HERE, name), "w") as f:
        json.dump(obj, f, indent=1)
    print("wrote", name)


def run_variant(bessel):
    _setup(bessel)
    import numpy as np

    if bessel == "ref":
        _dump("greens.json", gen_greens(np.random.default_rng(20261203)))
        _dump("long_4particle.json", gen_long_4(np.random.default_rng(20261204)))
        _dump("icm_energy.json", gen_icm(np.random.default_rng(20261205)))
        _dump("short_pair_refbessel.json",
              dict(source="test/Force_short_test.jl:9-93", cases=gen_short_pair(np.random.default_rng(20261206), "ref")))
    else:
        _dump("short_pair_accurate.json",
              dict(source="test/Force_short_test.jl:55-93 with accurate J0/J1",
                   cases=gen_short_pair(np.random.default_rng(20261206), "accurate")))
        _dump("system_python.json", gen_system(np.random.default_rng(20261207)))
        _dump("long_exact.json", gen_exact(np.random.default_rng(20261208)))
        _dump("long_ties.json", gen_ties(np.random.default_rng(20261209)))
        _dump("short_norm.json", gen_norm(np.random.default_rng(20261210)))


if __name__ == "__main__":
    variant = [a for a in sys.argv[1:] if a.startswith("--bessel=")]
    if variant:
        run_variant(variant[0].split("=", 1)[1])
    else:
        ref = os.path.dirname(os.path.dirname(REF_LIB))
        for v in ("ref", "accurate"):
            subprocess.run([sys.executable, os.path.abspath(__file__), f"--bessel={v}", f"--reference={ref}"],
                           check=True)
