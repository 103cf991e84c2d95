"""Config 5 stress: N = 1e6 (+-1), Lx = Ly = 3162, Lz = 10, gamma_up =
gamma_down = 0.99, alpha = 0.1, r_c = 10, P = 2000 (the near-singular
dielectric contrast where 1 - g_u g_d e^{-2 k L_z} loses digits).

* FP32+fix against FP64 on the GPU: relative L2 force error <= 1e-5 and
  energy error <= 1e-5 relative (the total is a sum of +-q_i q_j terms that
  cancel to about 1e-2 of their magnitude, which amplifies the FP32 node
  rounding: measured 1.1e-6); the per-particle error distribution is
  written as JSON to $QEM_STRESS_REPORT when that variable is set.
* FP64 GPU against the CPU oracle on sub-samples: short-range forces of the
  particles of a 150 x 150 window (the oracle evaluates the window plus an
  r_c halo; particles at least r_c inside compare) at <= 1e-11, and the long
  range for all N on a 32-vector subset of the k-set at <= 1e-8 (the oracle
  restates the reference's "total minus running sum" suffix sums,
  Force_long.jl:97-98, which lose digits in proportion to e^{k L_z}: about
  1e-9 .. 5e-9 for the larger k of a batch at L_z = 10).
"""
import json
import os

import numpy as np
import pytest

import oracle as O
from qem4molly_b200 import _lib as L
from qem4molly_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def stress():
    cfg = W.config5()
    e64 = W.engine_for(cfg, "fp64")
    e32 = W.engine_for(cfg, "fp32")
    k3, sK = e64.get_kset()
    e32.set_kset(k3, sK)
    F64, E64 = e64.forces(cfg["xyz"], cfg["q"], energy=True)
    F32, E32 = e32.forces(cfg["xyz"], cfg["q"], energy=True)
    return cfg, e64, F64, E64, F32, E32


def test_config5_fp32_vs_fp64_distribution(stress):
    cfg, _, F64, E64, F32, E32 = stress
    d = np.linalg.norm(F32 - F64, axis=1)
    n64 = np.linalg.norm(F64, axis=1)
    rms = np.sqrt(np.mean(n64 ** 2))
    per_rms = d / rms
    per_own = d / np.maximum(n64, 1e-300)
    l2 = float(np.linalg.norm(F32 - F64) / np.linalg.norm(F64))
    pct = [50, 90, 99, 99.9, 100]
    report = {
        "workload": "config5: N=1e6 +-1, Lx=Ly=3162, Lz=10, gamma_up=gamma_down=0.99, alpha=0.1, r_c=10, P=2000",
        "force_rel_l2": l2,
        "per_particle_err_over_rms": {f"p{p}": float(np.percentile(per_rms, p)) for p in pct},
        "per_particle_err_over_own": {f"p{p}": float(np.percentile(per_own, p)) for p in pct},
        "energy_fp64": E64, "energy_fp32": E32, "energy_rel_err": abs(E32 - E64) / abs(E64),
    }
    path = os.environ.get("QEM_STRESS_REPORT")
    if path:
        with open(path, "w") as f:
            json.dump(report, f, indent=1)
    assert l2 <= 1e-5, report
    assert report["energy_rel_err"] <= 1e-5, report


def test_config5_fp64_short_vs_oracle_window(stress):
    cfg, e64, _, _, _, _ = stress
    xyz, q = cfg["xyz"], cfg["q"]
    Fs = e64.forces(xyz, q, terms=L.QEM_TERM_SHORT)
    rc = cfg["r_cutoff"]
    x0, y0, w = 1000.0, 2000.0, 150.0
    inw = (xyz[:, 0] > x0 - rc) & (xyz[:, 0] < x0 + w + rc) & (xyz[:, 1] > y0 - rc) & (xyz[:, 1] < y0 + w + rc)
    idx = np.nonzero(inw)[0]
    p = O.params(cfg["L"], cfg["alpha"], rc, cfg["gamma_down"], cfg["gamma_up"], accuracy=cfg["accuracy"],
                 N_t=cfg["N_t"])
    Fo = O.short_forces(p, xyz[idx], q[idx])
    sub = xyz[idx]
    inner = (sub[:, 0] > x0 + rc) & (sub[:, 0] < x0 + w - rc) & (sub[:, 1] > y0 + rc) & (sub[:, 1] < y0 + w - rc)
    assert inner.sum() > 500
    assert W.rel_err(Fs[idx[inner]], Fo[inner])[0] <= 1e-11


def test_config5_fp64_long_vs_oracle_ksubset(stress):
    cfg, _, _, _, _, _ = stress
    e = W.engine_for(cfg, "fp64")
    k3, sK = e.get_kset()
    k3 = k3[:32]
    e.set_kset(k3, sK)
    F = e.forces(cfg["xyz"], cfg["q"], terms=L.QEM_TERM_LONG)
    p = O.params(cfg["L"], cfg["alpha"], cfg["r_cutoff"], cfg["gamma_down"], cfg["gamma_up"])
    Fo = O.F_long(p, cfg["xyz"], cfg["q"], k3, sK)
    assert W.rel_err(F, Fo)[0] <= 1e-8
