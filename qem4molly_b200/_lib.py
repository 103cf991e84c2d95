"""ctypes binding of libqem.so (the C-ABI declared in include/qem.h).

The shared library is the product: every force/energy evaluation runs in its
CUDA kernels.  There is no CPU fallback -- if the library is missing or no GPU
is present, calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
import re

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libqem.so")
HEADER = os.path.join(os.path.dirname(_PKG), "include", "qem.h")

QEM_OK = 0
STATUS = {0: "QEM_OK", 1: "QEM_ERR_ARG", 2: "QEM_ERR_OUT_OF_SLAB", 3: "QEM_ERR_NONFINITE",
          4: "QEM_ERR_NB_OVERFLOW", 5: "QEM_ERR_TIMEOUT", 6: "QEM_ERR_CUDA", 7: "QEM_ERR_NO_KSET",
          8: "QEM_ERR_RANGE"}
QEM_CUTOFF_PYTHON, QEM_DIR_MINIMAGE, QEM_PAIR_PHYSICAL = 0x1, 0x2, 0x4
QEM_STALE_NEIGHBORS, QEM_RESAMPLE_KSET, QEM_EQUAL_Z_TIES = 0x8, 0x10, 0x20
QEM_PYTHON_MODE = QEM_CUTOFF_PYTHON | QEM_DIR_MINIMAGE | QEM_PAIR_PHYSICAL
QEM_FP64, QEM_FP32_FIX = 0, 1
QEM_TERM_SHORT, QEM_TERM_LONG, QEM_TERM_LJ, QEM_TERM_ALL = 0x1, 0x2, 0x4, 0x7
QEM_MEM_HOST, QEM_MEM_DEVICE = 0, 1
QEM_BATCH_AUTO, QEM_BATCH_FUSED, QEM_BATCH_POOL = 0, 1, 2
QEM_NOALLOC_MAX_N, QEM_NOALLOC_MAX_P = 32768, 512
QEM_MAX_KSET = 1048560


class QemError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class LJWall(C.Structure):
    _fields_ = [("cutoff", C.c_double), ("sigma", C.c_double), ("eps", C.c_double),
                ("sub_pos", C.c_double), ("direction", C.c_double)]


class Params(C.Structure):
    _fields_ = [("Lx", C.c_double), ("Ly", C.c_double), ("Lz", C.c_double), ("alpha", C.c_double),
                ("r_cutoff", C.c_double), ("gamma_down", C.c_double), ("gamma_up", C.c_double),
                ("eps_0", C.c_double), ("accuracy", C.c_double), ("N_t", C.c_int32), ("rbe_p", C.c_int32),
                ("iter_period", C.c_int32), ("n_walls", C.c_int32), ("walls", LJWall * 2),
                ("mode_flags", C.c_uint32), ("precision", C.c_int32), ("device", C.c_int32),
                ("reserved0", C.c_int32), ("pv_eps", C.c_double), ("reserved", C.c_int32 * 2)]


_lib = None


def header_functions():
    """Names of the functions declared in include/qem.h."""
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(qem_[a-z_0-9]+)\s*\(", txt)))


def load(build: bool = False):
    """Load libqem.so (building it first when build=True)."""
    global _lib
    if _lib is not None:
        return _lib
    if build:
        from .build import build_lib

        build_lib()
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: run `python -m qem4molly_b200.build` (needs nvcc)")
    L = C.CDLL(LIB_PATH)
    vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int32)
    H = C.c_void_p
    PP = C.POINTER(Params)
    sig = {
        "qem_default_params": (None, [PP]),
        "qem_inter_params": (C.c_int32, [PP, C.c_int64, C.c_double, C.c_int32, C.c_int32]),
        "qem_create": (C.c_int32, [PP, C.POINTER(H)]),
        "qem_destroy": (None, [H]),
        "qem_last_error": (C.c_char_p, [H]),
        "qem_status_string": (C.c_char_p, [C.c_int32]),
        "qem_set_kset": (C.c_int32, [H, dp, C.c_int32, C.c_double]),
        "qem_sample_kset": (C.c_int32, [H, C.c_uint64, C.c_int32]),
        "qem_get_kset": (C.c_int32, [H, dp, C.c_int32, ip, dp]),
        "qem_kset_batch": (C.c_int32, [H, C.POINTER(C.c_uint64)]),
        "qem_draw_kset": (C.c_int32, [PP, C.c_uint64, C.c_uint64, C.c_int64, C.c_int32, dp, dp]),
        "qem_exact_kset_rows": (C.c_int32, [C.c_double, C.c_double, C.c_double, C.c_double, dp, dp, C.c_int64,
                                            C.POINTER(C.c_int64)]),
        "qem_set_kset_weighted": (C.c_int32, [H, dp, dp, C.c_int32]),
        "qem_set_kset_exact": (C.c_int32, [H, C.c_double, ip]),
        "qem_get_kset_weights": (C.c_int32, [H, dp, C.c_int32, ip]),
        "qem_forces": (C.c_int32, [H, C.c_int32, vp, vp, vp, dp, C.c_uint32, C.c_int32, vp]),
        "qem_short_forces": (C.c_int32, [H, C.c_int32, vp, vp, vp, C.c_int32, vp]),
        "qem_long_forces": (C.c_int32, [H, C.c_int32, vp, vp, vp, C.c_int32, vp]),
        "qem_lj_forces": (C.c_int32, [H, C.c_int32, vp, vp, C.c_int32, vp]),
        "qem_potential_energy": (C.c_int32, [H, C.c_int32, vp, vp, dp, C.c_uint32, C.c_int32, vp]),
        "qem_backward": (C.c_int32, [H, C.c_int32, vp, vp, vp, C.c_double, vp, vp, dp, C.c_uint32, C.c_int32, vp]),
        "qem_pair_list": (C.c_int32, [H, C.c_int32, dp, ip, C.c_int64, C.POINTER(C.c_int64)]),
        "qem_cell_index": (C.c_int32, [H, C.c_int32, dp, ip, ip, C.c_int32, ip, ip]),
        "qem_z_order": (C.c_int32, [H, C.c_int32, dp, ip]),
        "qem_set_profiling": (C.c_int32, [H, C.c_int32]),
        "qem_get_timings": (C.c_int32, [H, dp, C.c_int32, ip, C.c_char_p, C.c_int32]),
        "qem_get_counts": (C.c_int32, [H, C.POINTER(C.c_int64), C.c_int32]),
        "qem_version": (C.c_char_p, []),
        "qem_measure_peaks": (C.c_int32, [C.c_int32, dp, dp]),
        "qem_measure_fp64_peak": (C.c_int32, [C.c_int32, dp]),
        "qem_long_forces_noalloc": (C.c_int32, [PP, C.c_int32, vp, vp, C.c_int32, dp, C.c_double, vp, vp]),
        "qem_set_shard": (C.c_int32, [H, C.c_int32, C.c_int32]),
        "qem_batch_create": (C.c_int32, [C.c_int32, C.POINTER(H), ip, C.POINTER(vp)]),
        "qem_batch_destroy": (None, [vp]),
        "qem_batch_last_error": (C.c_char_p, [vp]),
        "qem_batch_forces": (C.c_int32, [vp, vp, vp, vp, C.c_uint32, vp]),
        "qem_batch_check": (C.c_int32, [vp, vp]),
        "qem_batch_md": (C.c_int32, [vp, C.c_int32, C.c_double, vp, vp, vp, vp, C.c_uint32, vp]),
        "qem_batch_autotune": (C.c_int32, [vp, vp, vp, vp, C.c_uint32, vp, ip, dp]),
        "qem_batch_set_thermostat": (C.c_int32, [vp, C.c_double, C.c_double, C.c_uint64]),
        "qem_batch_set_mode": (C.c_int32, [vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
        "qem_batch_get_mode": (C.c_int32, [vp, ip, ip, ip, ip, ip, C.POINTER(C.c_char_p)]),
        "qem_batch_thermostat_step": (C.c_int32, [vp, C.POINTER(C.c_uint64)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def default_params() -> Params:
    p = Params()
    load().qem_default_params(C.byref(p))
    return p
