"""ctypes wrapper of the FP64 CPU oracle (``qem_oracle.c``).

TEST INFRASTRUCTURE ONLY.  This module is the checker: the test-suite,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference arm
import it.  The product package ``qem4molly_b200`` never imports it and has no
CPU fallback through it.

Every function restates the reference's Julia semantics (file:line given in
``qem_oracle.c``); the energies follow the python_lib formulas because the
Julia package defines none.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libqem_oracle.so")
_lib = None

CUTOFF_JULIA, CUTOFF_PYTHON = 0, 1
DIR_RAW, DIR_MINIMAGE = 0, 1
PAIR_JULIA, PAIR_PHYSICAL = 0, 1


class Params(C.Structure):
    _fields_ = [
        ("Lx", C.c_double), ("Ly", C.c_double), ("Lz", C.c_double),
        ("alpha", C.c_double), ("r_cutoff", C.c_double),
        ("gamma_1", C.c_double), ("gamma_2", C.c_double),
        ("eps_0", C.c_double), ("accuracy", C.c_double),
        ("N_t", C.c_int), ("cutoff_mode", C.c_int),
        ("dir_mode", C.c_int), ("pair_mode", C.c_int), ("z_ties", C.c_int), ("pv_eps", C.c_double),
    ]


class Elem(C.Structure):
    _fields_ = [("a", C.c_double * 4), ("b", C.c_double * 4), ("sa", C.c_double * 4),
                ("kf1", C.c_double * 4), ("kf2", C.c_double * 4), ("rho", C.c_double)]


def build() -> str:
    """Compile the oracle shared library in place (make -C oracle)."""
    src = os.path.join(_HERE, "qem_oracle.c")
    if (not os.path.exists(_LIB_PATH)) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_LIB_PATH)
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int)
        P = C.POINTER(Params)
        E = C.POINTER(Elem)
        sig = {
            "qo_gauss_legendre": (C.c_int, [C.c_int, dp, dp]),
            "qo_elem_pair": (None, [P, C.c_double, C.c_double, C.c_double, E]),
            "qo_elem_self": (None, [P, C.c_double, E]),
            "qo_Gamma_1": (C.c_double, [P, C.c_double, E, C.c_int]),
            "qo_Gamma_2": (C.c_double, [P, C.c_double, E, C.c_int]),
            "qo_dz_Gamma_1": (C.c_double, [P, C.c_double, E, C.c_int]),
            "qo_dz_Gamma_2": (C.c_double, [P, C.c_double, E, C.c_int]),
            "qo_F_short_ij": (C.c_int, [P, C.c_double, C.c_double, dp, dp, C.c_int, dp]),
            "qo_F_short_i": (C.c_double, [P, C.c_double, dp, C.c_int]),
            "qo_pairs_bruteforce": (C.c_long, [P, C.c_int, dp, ip, C.c_long]),
            "qo_pairs_cells": (C.c_long, [P, C.c_int, dp, ip, C.c_long]),
            "qo_short_forces": (None, [P, C.c_int, dp, dp, C.c_long, ip, dp, C.c_int]),
            "qo_lj_forces": (C.c_int, [C.c_int, dp, C.c_double, C.c_double, C.c_double, C.c_double,
                                       C.c_double, dp]),
            "qo_kset_generator": (C.c_long, [C.c_double, C.c_double, C.c_double, C.c_double, dp,
                                             C.POINTER(C.c_float), dp, C.c_long]),
            "qo_sortperm_z": (None, [C.c_int, dp, ip]),
            "qo_Fl_non_sort": (None, [dp, C.c_int, dp, dp, C.c_double, C.c_double, C.c_double, dp,
                                      C.c_int]),
            "qo_Fl_sort": (None, [dp, C.c_int, ip, dp, dp, dp, C.c_int]),
            "qo_Flz_sort_k0": (None, [C.c_int, ip, dp, dp]),
            "qo_Flz_self": (None, [dp, C.c_int, dp, dp, C.c_double, C.c_double, C.c_double, dp]),
            "qo_F_l_total": (None, [P, dp, C.c_int, dp, dp, ip, dp, C.c_int]),
            "qo_F_long": (None, [P, C.c_int, dp, dp, ip, C.c_int, dp, C.c_double, dp, C.c_int]),
            "qo_energy_pair": (C.c_double, [P, C.c_double, C.c_double, dp, dp]),
            "qo_energy_self": (C.c_double, [P, C.c_double, dp]),
            "qo_energy_short": (C.c_double, [P, C.c_int, dp, dp, C.c_long, ip, C.c_int]),
            "qo_sigma_s": (C.c_double, [dp, C.c_int, dp, dp, C.c_double, C.c_double, C.c_double]),
            "qo_sigma_ns": (C.c_double, [dp, C.c_int, dp, dp, ip]),
            "qo_energy_k0": (C.c_double, [P, C.c_int, dp, dp, ip]),
            "qo_energy_long": (C.c_double, [P, C.c_int, dp, dp, ip, C.c_int, dp, C.c_double]),
            "qo_pairs_eval": (None, [P, dp, dp, C.c_long, ip, dp, C.c_int]),
            "qo_self_eval": (None, [P, C.c_int, dp, dp, dp, C.c_int]),
            "qo_max_threads": (C.c_int, []),
            "qo_exact_kset": (C.c_long, [C.c_double, C.c_double, C.c_double, C.c_double, dp, dp, C.c_long]),
            "qo_F_long_w": (None, [P, C.c_int, dp, dp, ip, C.c_int, dp, dp, dp, C.c_int]),
            "qo_energy_long_w": (C.c_double, [P, C.c_int, dp, dp, ip, C.c_int, dp, dp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _d(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(C.POINTER(C.c_double))


def _i(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(C.POINTER(C.c_int))


def params(L, alpha, r_cutoff, gamma_1=0.0, gamma_2=0.0, eps_0=1.0, accuracy=1e-6, N_t=30,
           cutoff_mode=CUTOFF_JULIA, dir_mode=DIR_RAW, pair_mode=PAIR_JULIA, z_ties=0, pv_eps=0.0) -> Params:
    """z_ties=1: equal-z particles are neither below nor above each other in the z-ordered sums
    (python_lib equal_cell, Sigma_Gamma_func_njit.py:168-281); 0: the plain sortperm order."""
    Lx, Ly, Lz = L
    return Params(float(Lx), float(Ly), float(Lz), float(alpha), float(r_cutoff), float(gamma_1),
                  float(gamma_2), float(eps_0), float(accuracy), int(N_t), int(cutoff_mode),
                  int(dir_mode), int(pair_mode), int(z_ties), float(pv_eps))


def gauss_legendre(n):
    x = np.zeros(n)
    w = np.zeros(n)
    lib().qo_gauss_legendre(n, _d(x)[1], _d(w)[1])
    return x, w


def elem_pair(p, z_i, z_j, rho):
    e = Elem()
    lib().qo_elem_pair(C.byref(p), z_i, z_j, rho, C.byref(e))
    return e


def elem_self(p, z_i):
    e = Elem()
    lib().qo_elem_self(C.byref(p), z_i, C.byref(e))
    return e


def Gamma_1(p, k, e, l=0):
    return lib().qo_Gamma_1(C.byref(p), k, C.byref(e), l)


def Gamma_2(p, k, e, l=0):
    return lib().qo_Gamma_2(C.byref(p), k, C.byref(e), l)


def dz_Gamma_1(p, k, e, l=0):
    return lib().qo_dz_Gamma_1(C.byref(p), k, C.byref(e), l)


def dz_Gamma_2(p, k, e, l=0):
    return lib().qo_dz_Gamma_2(C.byref(p), k, C.byref(e), l)


def F_short_ij(p, q_i, q_j, c_i, c_j, single=False):
    """Force on i from j (3) and the z-force on j from i as F_short_ij(j, i)."""
    out = np.zeros(4)
    ci, pi = _d(c_i)
    cj, pj = _d(c_j)
    lib().qo_F_short_ij(C.byref(p), q_i, q_j, pi, pj, int(single), _d(out)[1])
    return out[:3].copy(), out[3]


def F_short_i(p, q_i, c_i, single=False):
    ci, pi = _d(c_i)
    return np.array([0.0, 0.0, lib().qo_F_short_i(C.byref(p), q_i, pi, int(single))])


def pairs(p, xyz, method="auto"):
    xyz, px = _d(xyz)
    N = xyz.shape[0]
    f = lib().qo_pairs_bruteforce
    if method == "cells" or (method == "auto" and N > 3000):
        f = lib().qo_pairs_cells
    n = f(C.byref(p), N, px, None, 0)
    out = np.zeros((max(n, 1), 2), dtype=np.int32)
    f(C.byref(p), N, px, _i(out)[1], n)
    return out[:n]


def short_forces(p, xyz, q, pair_list=None, nthreads=0):
    xyz, px = _d(xyz)
    q, pq = _d(q)
    if pair_list is None:
        pair_list = pairs(p, xyz)
    pl, pp = _i(pair_list)
    F = np.zeros_like(xyz)
    lib().qo_short_forces(C.byref(p), xyz.shape[0], px, pq, pl.shape[0], pp, _d(F)[1], nthreads)
    return F


def lj_forces(xyz, cutoff, sigma, eps, sub_pos, direction, F=None):
    """Accumulates the wall force into F (z only); returns (F, n_out_of_slab)."""
    xyz, px = _d(xyz)
    if F is None:
        F = np.zeros_like(xyz)
    F, pf = _d(F)
    bad = lib().qo_lj_forces(xyz.shape[0], px, cutoff, sigma, eps, sub_pos, direction, pf)
    return F, bad


def kset_generator(Lx, Ly, alpha, accuracy):
    s = C.c_double()
    n = lib().qo_kset_generator(Lx, Ly, alpha, accuracy, None, None, C.byref(s), 0)
    K = np.zeros((n, 3))
    P = np.zeros(n, dtype=np.float32)
    lib().qo_kset_generator(Lx, Ly, alpha, accuracy, _d(K)[1], P.ctypes.data_as(C.POINTER(C.c_float)),
                            C.byref(s), n)
    return K, P, s.value


def sortperm_z(xyz):
    xyz, px = _d(xyz)
    z = np.zeros(xyz.shape[0], dtype=np.int32)
    lib().qo_sortperm_z(xyz.shape[0], px, _i(z)[1])
    return z


def Fl_non_sort(k3, xyz, q, g1, g2, Lz):
    xyz, px = _d(xyz)
    out = np.zeros_like(xyz)
    lib().qo_Fl_non_sort(_d(k3)[1], xyz.shape[0], px, _d(q)[1], g1, g2, Lz, _d(out)[1], 1)
    return out


def Fl_sort(k3, zlist, xyz, q):
    xyz, px = _d(xyz)
    out = np.zeros_like(xyz)
    lib().qo_Fl_sort(_d(k3)[1], xyz.shape[0], _i(zlist)[1], px, _d(q)[1], _d(out)[1], 1)
    return out


def Flz_sort_k0(zlist, q):
    q, pq = _d(q)
    out = np.zeros((q.shape[0], 3))
    lib().qo_Flz_sort_k0(q.shape[0], _i(zlist)[1], pq, _d(out)[1])
    return out


def Flz_self(k3, xyz, q, g1, g2, Lz):
    xyz, px = _d(xyz)
    out = np.zeros_like(xyz)
    lib().qo_Flz_self(_d(k3)[1], xyz.shape[0], px, _d(q)[1], g1, g2, Lz, _d(out)[1])
    return out


def F_l_total(p, k3, xyz, q, zlist):
    xyz, px = _d(xyz)
    out = np.zeros_like(xyz)
    lib().qo_F_l_total(C.byref(p), _d(k3)[1], xyz.shape[0], px, _d(q)[1], _i(zlist)[1], _d(out)[1], 1)
    return out


def F_long(p, xyz, q, kset, sum_K, zlist=None, nthreads=0):
    xyz, px = _d(xyz)
    kset, pk = _d(kset)
    F = np.zeros_like(xyz)
    zl = None if zlist is None else _i(zlist)[1]
    lib().qo_F_long(C.byref(p), xyz.shape[0], px, _d(q)[1], zl, kset.shape[0], pk, sum_K, _d(F)[1], nthreads)
    return F


def exact_kset(L, alpha, k_cutoff):
    """Exact-sum k-set (Force_long.jl:220-233, typos fixed): rows (kx, ky, k) of every
    lattice vector with 0 < k < k_cutoff in the Julia loop order, and weights e^{-k^2/4 alpha}."""
    n = lib().qo_exact_kset(L[0], L[1], alpha, k_cutoff, None, None, 0)
    k3 = np.zeros((n, 3))
    w = np.zeros(n)
    lib().qo_exact_kset(L[0], L[1], alpha, k_cutoff, _d(k3)[1], _d(w)[1], n)
    return k3, w


def F_long_weighted(p, xyz, q, kset, w, zlist=None, nthreads=0):
    """F_long with a per-k weight w[m] in place of sum_K / P (exact k-sum: w = e^{-k^2/4 alpha})."""
    xyz, px = _d(xyz)
    kset, pk = _d(kset)
    w, pw = _d(w)
    F = np.zeros_like(xyz)
    zl = None if zlist is None else _i(zlist)[1]
    lib().qo_F_long_w(C.byref(p), xyz.shape[0], px, _d(q)[1], zl, kset.shape[0], pk, pw, _d(F)[1], nthreads)
    return F


def energy_long_weighted(p, xyz, q, kset, w, zlist=None):
    xyz, px = _d(xyz)
    kset, pk = _d(kset)
    w, pw = _d(w)
    zl = None if zlist is None else _i(zlist)[1]
    return lib().qo_energy_long_w(C.byref(p), xyz.shape[0], px, _d(q)[1], zl, kset.shape[0], pk, pw)


def energy_short(p, xyz, q, pair_list=None, nthreads=0):
    xyz, px = _d(xyz)
    if pair_list is None:
        pair_list = pairs(p, xyz)
    pl, pp = _i(pair_list)
    return lib().qo_energy_short(C.byref(p), xyz.shape[0], px, _d(q)[1], pl.shape[0], pp, nthreads)


def energy_pair(p, q_i, q_j, c_i, c_j):
    return lib().qo_energy_pair(C.byref(p), q_i, q_j, _d(c_i)[1], _d(c_j)[1])


def energy_self(p, q_i, c_i):
    return lib().qo_energy_self(C.byref(p), q_i, _d(c_i)[1])


def sigma_s(k3, xyz, q, g1, g2, Lz):
    xyz, px = _d(xyz)
    return lib().qo_sigma_s(_d(k3)[1], xyz.shape[0], px, _d(q)[1], g1, g2, Lz)


def sigma_ns(k3, xyz, q, zlist):
    xyz, px = _d(xyz)
    return lib().qo_sigma_ns(_d(k3)[1], xyz.shape[0], px, _d(q)[1], _i(zlist)[1])


def energy_k0(p, xyz, q, zlist):
    xyz, px = _d(xyz)
    return lib().qo_energy_k0(C.byref(p), xyz.shape[0], px, _d(q)[1], _i(zlist)[1])


def energy_long(p, xyz, q, kset, sum_K, zlist=None):
    xyz, px = _d(xyz)
    kset, pk = _d(kset)
    zl = None if zlist is None else _i(zlist)[1]
    return lib().qo_energy_long(C.byref(p), xyz.shape[0], px, _d(q)[1], zl, kset.shape[0], pk, sum_K)


def lj_two_walls(xyz, walls):
    """Sum of Substrate_LJ forces for a list of wall dicts; returns (F, n_bad)."""
    F = np.zeros((np.asarray(xyz).shape[0], 3))
    bad = 0
    for w in walls:
        F, b = lj_forces(xyz, w["cutoff"], w["sigma"], w["eps"], w["sub_pos"], w["direction"], F)
        bad += b
    return F, bad


def pairs_eval(p, xyz, q, pair_list, nthreads=0):
    """F_short_ij rows (fx, fy, fz_i, fz_j) for the given pairs (timed CPU-baseline sample)."""
    xyz, px = _d(xyz)
    pl, pp = _i(pair_list)
    out = np.zeros((pl.shape[0], 4))
    lib().qo_pairs_eval(C.byref(p), px, _d(q)[1], pl.shape[0], pp, _d(out)[1], nthreads)
    return out


def self_eval(p, xyz, q, n, nthreads=0):
    xyz, px = _d(xyz)
    out = np.zeros(n)
    lib().qo_self_eval(C.byref(p), n, px, _d(q)[1], _d(out)[1], nthreads)
    return out


def max_threads():
    return lib().qo_max_threads()
