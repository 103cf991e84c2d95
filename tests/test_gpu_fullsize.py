"""The benchmark slab at full size against the FP64 oracle: N = 1e5 (+-1,
neutral), Lx = Ly = 1000, Lz = 10, z in [0.5, 9.5], gamma_up = gamma_down =
0.95, alpha = 0.1, r_c = 10, N_t = 30, P = 500, Julia semantics.  Every
ordered pair and self term of the short range, and the long range over all N
with the whole seeded k-set (about 15 s of oracle time on 16 host threads).

Tolerances (relative L2 over all particles):
  * FP64 path: short range <= 1e-11, long range and total <= 1e-9, energy
    <= 1e-10 relative;
  * FP32+fix path: total force <= 1e-5 (the benchmark metric's bound) and
    energy <= 1e-5 relative; the measured errors are printed.
"""
import numpy as np
import pytest

import oracle as O
from qem4molly_b200 import _lib as L
from qem4molly_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def slab():
    cfg = W.config2()
    e64 = W.engine_for(cfg, "fp64")
    e32 = W.engine_for(cfg, "fp32")
    k3, sK = e64.get_kset()
    e32.set_kset(k3, sK)
    p = O.params(cfg["L"], cfg["alpha"], cfg["r_cutoff"], cfg["gamma_down"], cfg["gamma_up"],
                 accuracy=cfg["accuracy"], N_t=cfg["N_t"])
    Fs = O.short_forces(p, cfg["xyz"], cfg["q"])
    Fl = O.F_long(p, cfg["xyz"], cfg["q"], k3, sK)
    return cfg, e64, e32, p, k3, sK, Fs, Fl


def test_fullsize_short_range_vs_oracle(slab):
    cfg, e64, e32, _, _, _, Fs, _ = slab
    F64 = e64.forces(cfg["xyz"], cfg["q"], terms=L.QEM_TERM_SHORT)
    F32 = e32.forces(cfg["xyz"], cfg["q"], terms=L.QEM_TERM_SHORT)
    r64, r32 = W.rel_err(F64, Fs), W.rel_err(F32, Fs)
    print(f"short range vs oracle: FP64 {r64[0]:.2e}, FP32+fix {r32[0]:.2e} (max/rms {r32[1]:.2e})")
    assert e64.counts()["pairs"] == 1_570_280
    assert r64[0] <= 1e-11
    assert r32[0] <= 1e-5


def test_fullsize_long_range_vs_oracle(slab):
    cfg, e64, e32, _, _, _, _, Fl = slab
    F64 = e64.forces(cfg["xyz"], cfg["q"], terms=L.QEM_TERM_LONG)
    F32 = e32.forces(cfg["xyz"], cfg["q"], terms=L.QEM_TERM_LONG)
    r64, r32 = W.rel_err(F64, Fl), W.rel_err(F32, Fl)
    print(f"long range vs oracle: FP64 {r64[0]:.2e}, FP32+fix {r32[0]:.2e}")
    assert r64[0] <= 1e-9
    assert r32[0] <= 1e-5


def test_fullsize_total_and_energy_vs_oracle(slab):
    """The benchmark's evaluation (short + self + long in one call) against
    the oracle: the metric's accuracy condition checked at the metric's size."""
    cfg, e64, e32, p, k3, sK, Fs, Fl = slab
    F64, E64 = e64.forces(cfg["xyz"], cfg["q"], energy=True)
    F32, E32 = e32.forces(cfg["xyz"], cfg["q"], energy=True)
    F32b = e32.forces(cfg["xyz"], cfg["q"])  # the energy-less kernels of the timed path
    Fo = Fs + Fl
    Eo = O.energy_short(p, cfg["xyz"], cfg["q"]) + O.energy_long(p, cfg["xyz"], cfg["q"], k3, sK)
    r64, r32, r32b = W.rel_err(F64, Fo), W.rel_err(F32, Fo), W.rel_err(F32b, Fo)
    print(f"total vs oracle: FP64 {r64[0]:.2e}, FP32+fix {r32[0]:.2e} / {r32b[0]:.2e}; energy FP64 "
          f"{abs(E64 - Eo) / abs(Eo):.2e}, FP32+fix {abs(E32 - Eo) / abs(Eo):.2e}")
    assert r64[0] <= 1e-9
    assert r32[0] <= 1e-5 and r32b[0] <= 1e-5
    assert abs(E64 - Eo) <= 1e-10 * abs(Eo)
    assert abs(E32 - Eo) <= 1e-5 * abs(Eo)
