"""C-ABI checks that need no GPU: the library loads, exports every function
include/qem.h declares, and the host-side parameter logic behaves."""
import ctypes as C

import numpy as np
import pytest

from qem4molly_b200 import _lib as L


@pytest.fixture(scope="module")
def lib():
    return L.load(build=True)


def test_exports_every_header_symbol(lib):
    names = L.header_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_version_names_sm100a(lib):
    assert b"sm_100a" in lib.qem_version()


def test_default_params_match_reference_defaults(lib):
    p = L.default_params()
    # QEM_short.jl:19 / QEM_long.jl:19 defaults
    assert p.eps_0 == 1.0 and p.accuracy == 1e-6 and p.N_t == 30 and p.rbe_p == 30 and p.iter_period == 100
    assert p.gamma_up == 0.0 and p.gamma_down == 0.0 and p.n_walls == 0 and p.precision == L.QEM_FP64


def test_qem_inter_params(lib):
    """Quasi_Ewald_Method.jl:5-16."""
    p = L.default_params()
    p.Lx, p.Ly, p.Lz = 100.0, 100.0, 50.0
    assert lib.qem_inter_params(C.byref(p), 1000, 1.0, 1, 10) == 0
    assert np.isclose(p.alpha, 1000 / 1e4) and np.isclose(p.r_cutoff, 1 / np.sqrt(0.1)) and p.rbe_p == 10
    assert lib.qem_inter_params(C.byref(p), 1000, 1.0, 0, 10) == 0
    assert np.isclose(p.alpha, np.sqrt(1000) / 1e4) and p.rbe_p == 0
    assert lib.qem_inter_params(C.byref(p), 0, 1.0, 1, 10) == 1


def _create(lib, **kw):
    p = L.default_params()
    p.Lx, p.Ly, p.Lz, p.alpha, p.r_cutoff = 100.0, 100.0, 10.0, 0.1, 10.0
    for k, v in kw.items():
        setattr(p, k, v)
    h = C.c_void_p()
    st = lib.qem_create(C.byref(p), C.byref(h))
    if st == 0:
        lib.qem_destroy(h)
    return st


@pytest.mark.parametrize("kw", [dict(r_cutoff=60.0), dict(alpha=0.0), dict(N_t=0), dict(N_t=65),
                                dict(accuracy=1.5), dict(gamma_up=1.0, gamma_down=1.0), dict(precision=7),
                                dict(mode_flags=0x100), dict(n_walls=3), dict(iter_period=0), dict(Lz=-1.0)])
def test_create_rejects_bad_params(lib, kw):
    assert _create(lib, **kw) == 1  # QEM_ERR_ARG before any CUDA call


def test_null_handle_calls_fail_cleanly(lib):
    assert lib.qem_forces(None, 0, None, None, None, None, 7, 0, None) == 1
    assert lib.qem_set_kset(None, None, 0, 0.0) == 1
    assert lib.qem_last_error(None) == b"NULL handle"
    assert lib.qem_status_string(2).startswith(b"particle run out")


def test_exact_kset_rows_match_oracle(lib):
    """qem_exact_kset_rows (host only) gives the oracle's exact-sum k-set, Force_long.jl:220-233
    with its typos fixed: same rows in the same order, weights exp(-k^2 / 4 alpha)."""
    import os
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
    import oracle as O

    for Lx, Ly, alpha, kc in [(12.0, 10.0, 0.8, 2.95), (100.0, 100.0, 0.1, 1.2), (37.0, 91.0, 0.3, 0.9)]:
        n = C.c_int64()
        dp = C.POINTER(C.c_double)
        assert lib.qem_exact_kset_rows(Lx, Ly, alpha, kc, None, None, 0, C.byref(n)) == 0
        k3 = np.zeros((n.value, 3))
        w = np.zeros(n.value)
        assert lib.qem_exact_kset_rows(Lx, Ly, alpha, kc, k3.ctypes.data_as(dp), w.ctypes.data_as(dp), n.value,
                                       C.byref(n)) == 0
        k3o, wo = O.exact_kset((Lx, Ly), alpha, kc)
        np.testing.assert_array_equal(k3, k3o)
        np.testing.assert_array_equal(w, wo)
    n = C.c_int64()
    assert lib.qem_exact_kset_rows(10.0, 10.0, 0.1, -1.0, None, None, 0, C.byref(n)) == 1
    assert lib.qem_exact_kset_rows(10.0, 10.0, 0.1, 1e9, None, None, 0, C.byref(n)) == 8  # QEM_ERR_RANGE
    assert lib.qem_set_kset_exact(None, 1.0, None) == 1


def test_params_layout_and_gamma_above_one_rules(lib):
    """qem_params is 200 bytes with pv_eps at offset 184; gamma_up * gamma_down > 1 needs FP64,
    python cutoffs, 0 < pv_eps < k_0 and non-empty sub-intervals (checked before any CUDA call)."""
    assert C.sizeof(L.Params) == 200 and L.Params.pv_eps.offset == 184
    e = float(np.exp(1.0))  # gamma_1 = gamma_2 = e: k_0 = ln(e^2) / (2 Lz) = 0.5 at Lz = 2
    base = dict(Lz=2.0, alpha=0.1, gamma_up=e, gamma_down=e)
    assert _create(lib, **base, mode_flags=L.QEM_PYTHON_MODE, pv_eps=0.0) == 1            # pv_eps missing
    assert _create(lib, **base, mode_flags=L.QEM_PYTHON_MODE, pv_eps=0.6) == 1            # pv_eps >= k_0
    assert _create(lib, **base, mode_flags=0, pv_eps=0.05) == 1                           # Julia cutoffs
    assert _create(lib, **base, mode_flags=L.QEM_PYTHON_MODE, pv_eps=0.05, precision=L.QEM_FP32_FIX) == 1
    assert _create(lib, **base, mode_flags=L.QEM_PYTHON_MODE, pv_eps=0.05, N_t=4) == 1     # N_1 = 0
    assert _create(lib, Lz=2.0, gamma_up=1.0, gamma_down=1.0) == 1                         # the pole at k = 0


# ---- the random-batch sampler (host restatement of the device draw) ----------
U64 = np.uint64


def _mix64(z):
    z = (z ^ (z >> U64(30))) * U64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> U64(27))) * U64(0x94D049BB133111EB)
    return z ^ (z >> U64(31))


def _draw64(seed, a, b, c):
    G = U64(0x9E3779B97F4A7C15)
    with np.errstate(over="ignore"):
        return _mix64(_mix64(_mix64(seed + G * (a + U64(1))) + G * (b + U64(1))) + G * (c + U64(1)))


def sampler_rows(Lx, Ly, alpha, accuracy, seed, n, row0, P):
    """numpy restatement of the library's batch draw: three SplitMix64 uniforms
    per row, the m_x != 0 / m_x = 0 part, then inverse CDFs (math.exp is the
    C library's exp, as in the library's tables)."""
    import math

    k_c = 2.0 * math.sqrt(-4.0 * alpha * math.log(accuracy))
    M = [int(math.ceil(k_c * L / (2.0 * math.pi))) + 1 for L in (Lx, Ly)]

    def cdf(Mi, L, skip0):
        c, out = 0.0, []
        for m in range(-Mi, Mi + 1):
            if skip0 and m == 0:
                continue
            k = 2.0 * math.pi * m / L
            c += math.exp(-k * k / (4.0 * alpha))
            out.append(c)
        return np.array(out)

    cxa, cxn, cya, cyn = cdf(M[0], Lx, False), cdf(M[0], Lx, True), cdf(M[1], Ly, False), cdf(M[1], Ly, True)
    Sx, Tx, Sy, Ty = cxn[-1], cxa[-1], cyn[-1], cya[-1]
    rows = np.arange(row0, row0 + P, dtype=U64)
    s = np.full(P, seed, dtype=U64)
    nn = np.full(P, n, dtype=U64)
    u = [(_draw64(s, nn, rows, np.full(P, j, dtype=U64)) >> U64(11)).astype(np.float64) * 2.0**-53 for j in range(3)]
    A = Sx * Ty
    partx = u[0] * (A + Sy) < A
    pick = lambda c, v: np.minimum(np.searchsorted(c, v, side="right"), len(c) - 1)
    ix = pick(cxn, u[1] * Sx)
    mx = np.where(partx, np.where(ix < M[0], ix - M[0], ix - M[0] + 1), 0)
    iy_all = pick(cya, u[2] * Ty) - M[1]
    iyn = pick(cyn, u[2] * Sy)
    my = np.where(partx, iy_all, np.where(iyn < M[1], iyn - M[1], iyn - M[1] + 1))
    kx = 2.0 * np.pi * mx.astype(np.float64) / Lx
    ky = 2.0 * np.pi * my.astype(np.float64) / Ly
    sum_K = Sx + Sy + Sx * Sy
    # support: Float32(exp(-k^2 / 4 alpha) / sum_K) > 0 (K_set_generator.jl:43);
    # the library draws an off-support row again from the next counter words,
    # which these parameters never need (such a row has probability < 2^-150)
    k2max = 4.0 * alpha * (150.0 * math.log(2.0) - math.log(sum_K))
    fx, fy = 2.0 * np.pi * mx / Lx, 2.0 * np.pi * my / Ly
    assert np.all(fx * fx + fy * fy < k2max)
    return np.stack([kx, ky, np.sqrt(kx * kx + ky * ky)], 1), sum_K


def _draw(lib, Lx, Ly, alpha, seed, n, row0, P, accuracy=1e-6):
    p = L.default_params()
    p.Lx, p.Ly, p.alpha, p.accuracy = Lx, Ly, alpha, accuracy
    k3 = np.zeros((max(P, 1), 3))
    sK = C.c_double()
    assert lib.qem_draw_kset(C.byref(p), seed, n, row0, P, k3.ctypes.data_as(C.POINTER(C.c_double)),
                             C.byref(sK)) == 0
    return k3[:P], sK.value


@pytest.mark.parametrize("Lx,Ly,alpha", [(1000.0, 1000.0, 0.1), (30.0, 45.0, 0.1), (5.0, 400.0, 0.02)])
def test_draw_kset_equals_its_restatement(lib, Lx, Ly, alpha):
    """qem_draw_kset (the host copy of the device draw) against an independent
    numpy restatement, bit for bit, for several batches and row offsets; sum_K
    is K_set_generator.jl:28."""
    import os
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
    import oracle as O

    for seed, n, row0 in [(7, 0, 0), (7, 1, 0), (123456789, 41, 250), (2**63 + 5, 2**40, 3)]:
        k3, sK = _draw(lib, Lx, Ly, alpha, seed, n, row0, 500)
        r3, rsK = sampler_rows(Lx, Ly, alpha, 1e-6, seed, n, row0, 500)
        np.testing.assert_array_equal(k3, r3)
        assert sK == rsK
    assert np.isclose(sK, O.kset_generator(Lx, Ly, alpha, 1e-6)[2], rtol=1e-12)
    a, _ = _draw(lib, Lx, Ly, alpha, 7, 0, 0, 300)
    b, _ = _draw(lib, Lx, Ly, alpha, 7, 1, 0, 300)
    c, _ = _draw(lib, Lx, Ly, alpha, 7, 0, 100, 200)
    assert not np.array_equal(a, b)
    np.testing.assert_array_equal(a[100:], c)
    assert np.all(a[:, 2] > 0)


def test_draw_kset_distribution(lib):
    """The draws follow exp(-k^2 / 4 alpha) / sum_K on the lattice without k = 0
    (K_set_generator.jl:30-41): chi-square against the oracle's table."""
    import os
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
    import oracle as O

    Lx = Ly = 30.0
    k3, _ = _draw(lib, Lx, Ly, 0.1, 99, 3, 0, 200_000)
    K, P, _ = O.kset_generator(Lx, Ly, 0.1, 1e-6)
    m = np.rint(k3[:, :2] * Lx / (2 * np.pi)).astype(int)
    assert not np.any((m[:, 0] == 0) & (m[:, 1] == 0))
    mref = np.rint(K[:, :2] * Lx / (2 * np.pi)).astype(int)
    key = lambda a: a[:, 0] * 1000 + a[:, 1]
    pref = dict(zip(key(mref), P.astype(np.float64)))
    vals, cnt = np.unique(key(m), return_counts=True)
    expected = np.array([pref[v] for v in vals]) * len(m)
    sel = expected > 50
    chi2 = np.sum((cnt[sel] - expected[sel]) ** 2 / expected[sel])
    assert chi2 / sel.sum() < 1.5
    # the mass of the rare cells is right too
    assert abs(cnt[~sel].sum() - expected[~sel].sum()) < 5 * np.sqrt(max(expected[~sel].sum(), 1.0)) + 5
