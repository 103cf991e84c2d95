"""Python mirror of QEM4Molly's interaction API, backed by libqem.so.

Names, keyword defaults and argument meaning follow the Julia package:

    QEM_short(L, r_cutoff, alpha; iter_period=100, gamma_1=0, gamma_2=0,
              eps_0=1, accuracy=1e-6, N_t=30)            src/QEM_short.jl:19-25
    QEM_long(L; k_cutoff=1.0, z_list=[], gamma_1=0, gamma_2=0, eps_0=1,
             accuracy=1e-6, alpha=1, rbe_mode=true, rbe_p=30) src/QEM_long.jl:19-30
    QEM_inter(n_atoms, L; s=1.0, accuracy=1e-6, rbe_mode=true, rbe_p=30,
              eps_0=1.0, gamma_1=0.0, gamma_2=0.0, N_t=30, iter_period=100)
                                                          src/Quasi_Ewald_Method.jl:3-24
    Substrate_LJ(; cutoff=1.0, sigma=0.5, eps=1.0, sub_pos=0.0, direction=+1)
                                                          src/Substrate_LJ.jl:15-17
    forces(inter, sys)  ==  Molly.forces(inter, sys, neighbors)

`sys` is any object with `coords` (N x 3) and `charges` (N) -- the fields the
reference reads from Molly's System (sys.coords, sys.atoms[i].charge).  The
gamma_1 / gamma_2 names are the reference's: gamma_1 is the lower (z = 0)
dielectric jump, gamma_2 the upper one.

Extra keywords (not in the reference): `precision` ("fp64" or "fp32"),
`mode` ("julia" = reference semantics, "python" = python_lib conventions),
`seed` for the random-batch sampler, `device`.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from . import _lib as _qem  # the constructors below take the reference's argument `L` (the box)


def _mode_flags(mode: str) -> int:
    if mode == "julia":
        return 0
    if mode == "python":
        return L.QEM_PYTHON_MODE
    raise ValueError("mode must be 'julia' or 'python'")


def _precision(precision: str) -> int:
    return {"fp64": L.QEM_FP64, "fp32": L.QEM_FP32_FIX}[precision]


class Engine:
    """One libqem handle: a configured QEM short + long + wall evaluator."""

    def __init__(self, *, L_box, alpha, r_cutoff, gamma_1=0.0, gamma_2=0.0, eps_0=1.0, accuracy=1e-6,
                 N_t=30, rbe_p=30, iter_period=100, walls=(), mode_flags=0, precision=L.QEM_FP64, device=0,
                 pv_eps=0.0):
        """pv_eps: window half-width of the regularised quadrature for gamma_1 * gamma_2 > 1."""
        lib = L.load()
        p = L.default_params()
        p.Lx, p.Ly, p.Lz = (float(v) for v in L_box)
        p.alpha, p.r_cutoff = float(alpha), float(r_cutoff)
        p.gamma_down, p.gamma_up = float(gamma_1), float(gamma_2)
        p.eps_0, p.accuracy = float(eps_0), float(accuracy)
        p.N_t, p.rbe_p, p.iter_period = int(N_t), int(rbe_p), int(iter_period)
        p.n_walls = len(walls)
        for i, w in enumerate(walls):
            p.walls[i] = L.LJWall(float(w.cutoff), float(w.sigma), float(w.eps), float(w.sub_pos),
                                  float(w.direction))
        p.mode_flags = int(mode_flags)
        p.precision = int(precision)
        p.device = int(device)
        p.pv_eps = float(pv_eps)
        self.params = p
        h = C.c_void_p()
        st = lib.qem_create(C.byref(p), C.byref(h))
        if st != 0:
            raise L.QemError(st, "qem_create failed (see stderr for the parameter that was rejected)")
        self._h = h
        self._lib = lib

    def close(self):
        if getattr(self, "_h", None):
            self._lib.qem_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st != 0:
            raise L.QemError(st, self._lib.qem_last_error(self._h).decode())

    def set_shard(self, rank, world):
        """Evaluate this rank's share of one system (see qem_set_shard); the W
        ranks' forces and energies sum to the unsharded result."""
        self._check(self._lib.qem_set_shard(self._h, int(rank), int(world)))

    # -- k-set -----------------------------------------------------------------
    def set_kset(self, k3, sum_K):
        k3 = np.ascontiguousarray(k3, dtype=np.float64).reshape(-1, 3)
        self._check(self._lib.qem_set_kset(self._h, k3.ctypes.data_as(C.POINTER(C.c_double)), k3.shape[0],
                                           float(sum_K)))

    def sample_kset(self, seed, P):
        self._check(self._lib.qem_sample_kset(self._h, int(seed) & 0xFFFFFFFFFFFFFFFF, int(P)))

    def set_kset_weighted(self, k3, w):
        """k-set rows (kx, ky, |k|) with a weight per row in place of sum_K / P."""
        k3 = np.ascontiguousarray(k3, dtype=np.float64).reshape(-1, 3)
        w = np.ascontiguousarray(w, dtype=np.float64).reshape(-1)
        if w.shape[0] != k3.shape[0]:
            raise ValueError("one weight per k-vector")
        self._check(self._lib.qem_set_kset_weighted(self._h, k3.ctypes.data_as(C.POINTER(C.c_double)),
                                                    w.ctypes.data_as(C.POINTER(C.c_double)), k3.shape[0]))

    def set_kset_exact(self, k_cutoff):
        """Exact (non-random-batch) k-sum: every lattice k with 0 < |k| < k_cutoff, weight
        exp(-k^2 / 4 alpha) (Force_long.jl:220-233).  Returns the number of k-vectors."""
        P = C.c_int32()
        self._check(self._lib.qem_set_kset_exact(self._h, float(k_cutoff), C.byref(P)))
        return P.value

    def get_kset_weights(self):
        """Per-row weights of a weighted k-set, or None for uniform sum_K / P weights."""
        P = C.c_int32()
        self._check(self._lib.qem_get_kset_weights(self._h, None, 0, C.byref(P)))
        if P.value == 0:
            return None
        w = np.zeros(P.value)
        self._check(self._lib.qem_get_kset_weights(self._h, w.ctypes.data_as(C.POINTER(C.c_double)), P.value,
                                                   C.byref(P)))
        return w

    def get_kset(self):
        P = C.c_int32()
        s = C.c_double()
        self._check(self._lib.qem_get_kset(self._h, None, 0, C.byref(P), C.byref(s)))
        out = np.zeros((max(P.value, 1), 3))
        self._check(self._lib.qem_get_kset(self._h, out.ctypes.data_as(C.POINTER(C.c_double)), P.value, None,
                                           None))
        return out[:P.value], s.value

    # -- evaluation ------------------------------------------------------------
    def forces(self, xyz, q, terms=L.QEM_TERM_ALL, energy=False, out=None):
        """Host arrays in, host arrays out.  Returns F (N x 3) or (F, E); `out` may be a
        preallocated (e.g. pinned) float64 N x 3 array that receives the forces."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        q = np.ascontiguousarray(q, dtype=np.float64).reshape(-1)
        if q.shape[0] != xyz.shape[0]:
            raise ValueError("coords and charges differ in length")
        if out is not None:
            if out.shape != xyz.shape or out.dtype != np.float64 or not out.flags.c_contiguous:
                raise ValueError("out must be a contiguous float64 array shaped like xyz")
            F = out
        else:
            F = np.zeros_like(xyz)
        E = C.c_double(0.0)
        st = self._lib.qem_forces(self._h, xyz.shape[0], xyz.ctypes.data, q.ctypes.data, F.ctypes.data,
                                  C.byref(E) if energy else None, int(terms), L.QEM_MEM_HOST, None)
        self._check(st)
        return (F, E.value) if energy else F

    def forces_device(self, xyz, q, F, terms=L.QEM_TERM_ALL, energy=False, stream=None):
        """torch CUDA tensors (float64, contiguous) in place; returns the energy or None."""
        import torch

        for t in (xyz, q, F):
            if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
                raise ValueError("device tensors must be contiguous float64 CUDA tensors")
        s = stream if stream is not None else torch.cuda.current_stream(xyz.device).cuda_stream
        E = C.c_double(0.0)
        st = self._lib.qem_forces(self._h, q.shape[0], C.c_void_p(xyz.data_ptr()), C.c_void_p(q.data_ptr()),
                                  C.c_void_p(F.data_ptr()), C.byref(E) if energy else None, int(terms),
                                  L.QEM_MEM_DEVICE, C.c_void_p(s))
        self._check(st)
        return E.value if energy else None

    def backward(self, xyz, q, gF=None, gE=0.0, terms=L.QEM_TERM_ALL):
        """Adjoint of forces() for L = gE * E + sum_i gF_i . F_i (host arrays, FP64).

        Returns (dL/dxyz (N x 3), dL/dq (N,), dL/d(gamma_1, gamma_2) (2,))."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        q = np.ascontiguousarray(q, dtype=np.float64).reshape(-1)
        if q.shape[0] != xyz.shape[0]:
            raise ValueError("coords and charges differ in length")
        g = None
        if gF is not None:
            g = np.ascontiguousarray(gF, dtype=np.float64).reshape(-1, 3)
            if g.shape != xyz.shape:
                raise ValueError("gF must be shaped like xyz")
        gx = np.zeros_like(xyz)
        gq = np.zeros_like(q)
        gg = (C.c_double * 2)()
        st = self._lib.qem_backward(self._h, xyz.shape[0], xyz.ctypes.data, q.ctypes.data,
                                    g.ctypes.data if g is not None else None, float(gE), gx.ctypes.data,
                                    gq.ctypes.data, gg, int(terms), L.QEM_MEM_HOST, None)
        self._check(st)
        return gx, gq, np.array([gg[0], gg[1]])

    def backward_device(self, xyz, q, gF, gE, gxyz, gq=None, terms=L.QEM_TERM_ALL, stream=None):
        """Device version of backward(): torch CUDA float64 tensors, gxyz / gq written in
        place (gF and gq may be None); returns dL/d(gamma_1, gamma_2) as a numpy array."""
        import torch

        for t in (xyz, q, gF, gxyz, gq):
            if t is not None and not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
                raise ValueError("device tensors must be contiguous float64 CUDA tensors")
        s = stream if stream is not None else torch.cuda.current_stream(xyz.device).cuda_stream
        gg = (C.c_double * 2)()
        ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None
        st = self._lib.qem_backward(self._h, q.shape[0], ptr(xyz), ptr(q), ptr(gF), float(gE), ptr(gxyz), ptr(gq),
                                    gg, int(terms), L.QEM_MEM_DEVICE, C.c_void_p(s))
        self._check(st)
        return np.array([gg[0], gg[1]])

    def energy(self, xyz, q, terms=L.QEM_TERM_SHORT | L.QEM_TERM_LONG):
        return self.forces(xyz, q, terms=terms, energy=True)[1]

    def pair_list(self, xyz):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        n = C.c_int64()
        dp = xyz.ctypes.data_as(C.POINTER(C.c_double))
        self._check(self._lib.qem_pair_list(self._h, xyz.shape[0], dp, None, 0, C.byref(n)))
        out = np.zeros((max(n.value, 1), 2), dtype=np.int32)
        self._check(self._lib.qem_pair_list(self._h, xyz.shape[0], dp, out.ctypes.data_as(C.POINTER(C.c_int32)),
                                            n.value, C.byref(n)))
        return out[:n.value]

    def cell_index(self, xyz):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        ncx, ncy = C.c_int32(), C.c_int32()
        self._check(self._lib.qem_cell_index(self._h, 0, xyz.ctypes.data_as(C.POINTER(C.c_double)), None, None, 0,
                                             C.byref(ncx), C.byref(ncy)))
        cell = np.zeros(xyz.shape[0], dtype=np.int32)
        start = np.zeros(ncx.value * ncy.value + 1, dtype=np.int32)
        ip = C.POINTER(C.c_int32)
        self._check(self._lib.qem_cell_index(self._h, xyz.shape[0], xyz.ctypes.data_as(C.POINTER(C.c_double)),
                                             cell.ctypes.data_as(ip), start.ctypes.data_as(ip), start.shape[0],
                                             C.byref(ncx), C.byref(ncy)))
        return cell, start, (ncx.value, ncy.value)

    def z_order(self, xyz):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        z = np.zeros(xyz.shape[0], dtype=np.int32)
        self._check(self._lib.qem_z_order(self._h, xyz.shape[0], xyz.ctypes.data_as(C.POINTER(C.c_double)),
                                          z.ctypes.data_as(C.POINTER(C.c_int32))))
        return z

    def set_profiling(self, on=True):
        self._check(self._lib.qem_set_profiling(self._h, 1 if on else 0))

    def timings(self):
        ms = (C.c_double * 32)()
        n = C.c_int32()
        names = C.create_string_buffer(1024)
        self._check(self._lib.qem_get_timings(self._h, ms, 32, C.byref(n), names, 1024))
        keys = names.value.decode().split(",") if n.value else []
        return dict(zip(keys, list(ms)[: n.value]))

    def counts(self):
        c = (C.c_int64 * 4)()
        self._check(self._lib.qem_get_counts(self._h, c, 4))
        return dict(pairs=c[0], particles=c[1], kvectors=c[2], launches=c[3])


@dataclass
class Substrate_LJ:
    """Substrate_LJ(; cutoff=1.0, sigma=0.5, eps=1.0, sub_pos=0.0, direction=+1)  (Substrate_LJ.jl:15)"""

    cutoff: float = 1.0
    sigma: float = 0.5
    eps: float = 1.0
    sub_pos: float = 0.0
    direction: int = +1


class QEM_short:
    """QEM_short(L, r_cutoff, alpha; ...)  (QEM_short.jl:19-25).  Mutable n_steps as in the reference."""

    def __init__(self, L, r_cutoff, alpha, *, iter_period=100, gamma_1=0, gamma_2=0, eps_0=1, accuracy=1e-6,
                 N_t=30, precision="fp64", mode="julia", stale_neighbors=False, device=0):
        self.L, self.r_cutoff, self.alpha = tuple(L), r_cutoff, alpha
        self.iter_period, self.gamma_1, self.gamma_2 = iter_period, gamma_1, gamma_2
        self.eps_0, self.accuracy, self.N_t = eps_0, accuracy, N_t
        self.n_steps = 0
        flags = _mode_flags(mode) | (_qem.QEM_STALE_NEIGHBORS if stale_neighbors else 0)
        self.engine = Engine(L_box=self.L, alpha=alpha, r_cutoff=r_cutoff, gamma_1=gamma_1, gamma_2=gamma_2,
                             eps_0=eps_0, accuracy=accuracy, N_t=N_t, rbe_p=0, iter_period=iter_period,
                             mode_flags=flags, precision=_precision(precision), device=device)


class QEM_long:
    """QEM_long(L; k_cutoff, z_list, gamma_1, gamma_2, eps_0, accuracy, alpha, rbe_mode, rbe_p)
    (QEM_long.jl:19-30).  rbe_mode=True: a fresh random batch of rbe_p k-vectors is drawn on every
    forces call, as Force_long.jl:235 does (pass `resample=False` to keep one batch).
    rbe_mode=False: the exact k-sum of Force_long.jl:220-233 (typos fixed) over every lattice k with
    0 < |k| < k_cutoff, weighted by exp(-k^2 / 4 alpha)."""

    def __init__(self, L, *, k_cutoff=1.0, z_list=(), gamma_1=0, gamma_2=0, eps_0=1, accuracy=1e-6, alpha=1,
                 rbe_mode=True, rbe_p=30, precision="fp64", mode="julia", seed=0, resample=True, device=0):
        self.L, self.k_cutoff, self.z_list = tuple(L), k_cutoff, list(z_list)
        self.gamma_1, self.gamma_2, self.eps_0, self.accuracy = gamma_1, gamma_2, eps_0, accuracy
        self.alpha, self.rbe_mode, self.rbe_p = alpha, rbe_mode, rbe_p
        flags = _mode_flags(mode) | (_qem.QEM_RESAMPLE_KSET if (resample and rbe_mode) else 0)
        # the short-range cutoff is irrelevant for the long range; any value < L/2 is valid
        self.engine = Engine(L_box=self.L, alpha=alpha, r_cutoff=0.25 * min(self.L[0], self.L[1]),
                             gamma_1=gamma_1, gamma_2=gamma_2, eps_0=eps_0, accuracy=accuracy,
                             rbe_p=rbe_p if rbe_mode else 0, mode_flags=flags, precision=_precision(precision),
                             device=device)
        if rbe_mode:
            self.engine.sample_kset(seed, rbe_p)
        else:
            self.n_k = self.engine.set_kset_exact(k_cutoff)


def QEM_inter(n_atoms, L, *, s=1.0, accuracy=1e-6, rbe_mode=True, rbe_p=30, eps_0=1.0, gamma_1=0.0, gamma_2=0.0,
              N_t=30, iter_period=100, **kw):
    """Quasi_Ewald_Method.jl:3-24: alpha = N / (Lx Ly), r_c = s / sqrt(alpha), k_c = 2 s sqrt(alpha)."""
    Lx, Ly, _ = L
    alpha = n_atoms / (Lx * Ly) if rbe_mode else np.sqrt(n_atoms) / (Lx * Ly)
    r_cutoff = s / np.sqrt(alpha)
    k_cutoff = 2 * s * np.sqrt(alpha)
    short = QEM_short(L, r_cutoff, alpha, iter_period=iter_period, gamma_1=gamma_1, gamma_2=gamma_2, eps_0=eps_0,
                      accuracy=accuracy, N_t=N_t, **{k: v for k, v in kw.items() if k != "seed"})
    long = QEM_long(L, k_cutoff=k_cutoff, gamma_1=gamma_1, gamma_2=gamma_2, eps_0=eps_0, accuracy=accuracy,
                    alpha=alpha, rbe_mode=rbe_mode, rbe_p=rbe_p if rbe_mode else 0, **kw)
    return short, long


@dataclass
class System:
    """Minimal stand-in for the parts of Molly's System the interactions read."""

    coords: np.ndarray
    charges: np.ndarray


class Batch:
    """Independent systems evaluated together (qem_batch_* of libqem): one Engine
    per system, device arrays laid end to end (system s owns particles
    [off[s], off[s] + N[s])).  Keeps its engines alive."""

    def __init__(self, engines, N):
        self._lib = L.load()
        self.engines = list(engines)
        self.N = [int(n) for n in N]
        if len(self.N) != len(self.engines):
            raise ValueError("one particle count per engine")
        self.off = np.concatenate([[0], np.cumsum(self.N)[:-1]]).astype(np.int64)
        hs = (C.c_void_p * len(self.engines))(*[e._h.value for e in self.engines])
        ns = (C.c_int32 * len(self.N))(*self.N)
        b = C.c_void_p()
        st = self._lib.qem_batch_create(len(self.engines), hs, ns, C.byref(b))
        if st != 0:
            raise L.QemError(st, "qem_batch_create failed")
        self._b = b

    def close(self):
        if getattr(self, "_b", None):
            self._lib.qem_batch_destroy(self._b)
            self._b = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st != 0:
            raise L.QemError(st, self._lib.qem_batch_last_error(self._b).decode())

    @staticmethod
    def _ptr(t):
        import torch

        if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
            raise ValueError("device tensors must be contiguous float64 CUDA tensors")
        return C.c_void_p(t.data_ptr())

    @staticmethod
    def _stream(t, stream):
        import torch

        return C.c_void_p(stream if stream is not None else torch.cuda.current_stream(t.device).cuda_stream)

    def forces(self, xyz, q, F, terms=L.QEM_TERM_ALL, stream=None):
        """Batched forces into F (asynchronous after the first call; see check())."""
        self._check(self._lib.qem_batch_forces(self._b, self._ptr(xyz), self._ptr(q), self._ptr(F), int(terms),
                                               self._stream(xyz, stream)))

    def check(self, stream=None):
        """Synchronises the stream and raises on any device status recorded since the last check."""
        import torch

        s = C.c_void_p(stream if stream is not None else torch.cuda.current_stream().cuda_stream)
        self._check(self._lib.qem_batch_check(self._b, s))

    def md(self, nsteps, dt, xyz, v, q, F, terms=L.QEM_TERM_ALL, stream=None):
        """nsteps graph-replayed velocity-Verlet steps (unit masses) in place."""
        self._check(self._lib.qem_batch_md(self._b, int(nsteps), float(dt), self._ptr(xyz), self._ptr(v),
                                           self._ptr(q), self._ptr(F), int(terms), self._stream(xyz, stream)))

    def set_thermostat(self, kT, nu, seed=0):
        """Andersen thermostat of the MD steps (Molly AndersenThermostat(temp, coupling_const),
        nu = 1 / coupling_const; unit masses); kT = 0 or nu = 0 switches it off."""
        self._check(self._lib.qem_batch_set_thermostat(self._b, float(kT), float(nu), int(seed) & (2**64 - 1)))

    def thermostat_step(self):
        """Number of thermostatted steps since the last set_thermostat."""
        n = C.c_uint64()
        self._check(self._lib.qem_batch_thermostat_step(self._b, C.byref(n)))
        return n.value

    def autotune(self, xyz, q, F, terms=L.QEM_TERM_ALL, stream=None):
        """Times the stream-pool widths and the fused tilings and keeps the fastest;
        returns (pool width or 0 for the fused phases, ms per batch evaluation)."""
        w = C.c_int32()
        ms = C.c_double()
        self._check(self._lib.qem_batch_autotune(self._b, self._ptr(xyz), self._ptr(q), self._ptr(F), int(terms),
                                                 self._stream(xyz, stream), C.byref(w), C.byref(ms)))
        return w.value, ms.value

    def set_mode(self, mode=L.QEM_BATCH_AUTO, ks=0, order=0, chunk=0):
        """QEM_BATCH_AUTO / _FUSED / _POOL; ks: k-slices per system of the fused force
        pass (0: each engine's own); order: 0 batch order, 1 largest system first;
        chunk: particles per chunk of the fused k-space passes (0: 512)."""
        self._check(self._lib.qem_batch_set_mode(self._b, int(mode), int(ks), int(order), int(chunk)))

    def mode(self):
        """dict(mode, ks, order, chunk, launches, why) of the way evaluations run now."""
        m, ks, order, ch, n = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        why = C.c_char_p()
        self._check(self._lib.qem_batch_get_mode(self._b, C.byref(m), C.byref(ks), C.byref(order), C.byref(ch),
                                                 C.byref(n), C.byref(why)))
        name = {L.QEM_BATCH_FUSED: "fused", L.QEM_BATCH_POOL: "pool"}.get(m.value, m.value)
        return dict(mode=name, ks=ks.value, order=order.value, chunk=ch.value, launches=n.value,
                    why=(why.value or b"").decode())


def forces(inter, sys, neighbors=None):
    """Molly.forces(inter, sys, neighbors) for QEM_short / QEM_long / Substrate_LJ (N x 3)."""
    xyz, q = np.asarray(sys.coords, dtype=np.float64), np.asarray(sys.charges, dtype=np.float64)
    if isinstance(inter, QEM_short):
        inter.n_steps += 1
        return inter.engine.forces(xyz, q, terms=L.QEM_TERM_SHORT)
    if isinstance(inter, QEM_long):
        return inter.engine.forces(xyz, q, terms=L.QEM_TERM_LONG)
    if isinstance(inter, Substrate_LJ):
        e = _wall_engine(inter, xyz)
        return e.forces(xyz, np.zeros(len(xyz)), terms=L.QEM_TERM_LJ)
    raise TypeError(f"no forces for {type(inter).__name__}")


def potential_energy(inter, sys, neighbors=None):
    """Molly.potential_energy for the QEM interactions (python_lib energy formulas)."""
    xyz, q = np.asarray(sys.coords, dtype=np.float64), np.asarray(sys.charges, dtype=np.float64)
    if isinstance(inter, QEM_short):
        return inter.engine.energy(xyz, q, terms=L.QEM_TERM_SHORT)
    if isinstance(inter, QEM_long):
        return inter.engine.energy(xyz, q, terms=L.QEM_TERM_LONG)
    raise TypeError(f"no potential energy for {type(inter).__name__} (the reference defines none)")


_WALL_ENGINES: dict = {}


def _wall_engine(w: Substrate_LJ, xyz):
    key = (w.cutoff, w.sigma, w.eps, w.sub_pos, w.direction)
    e = _WALL_ENGINES.get(key)
    if e is None:
        # the box does not enter the wall force (Substrate_LJ.jl:34-43); any valid box works
        e = Engine(L_box=(100.0, 100.0, 1.0), alpha=1.0, r_cutoff=1.0, walls=[w], rbe_p=0)
        _WALL_ENGINES[key] = e
    return e
