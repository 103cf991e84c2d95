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
