#!/usr/bin/env python
"""QEM force evaluations per second at N = 1e5 on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step" = one force evaluation of the whole system): the N = 1e5
slab of the benchmark configuration -- +-1 charges, Lx = Ly = 1000, Lz = 10,
gamma_up = gamma_down = 0.95, alpha = 0.1, r_c = 10, 30-node Gauss-Legendre
quadrature, P = 500 random-batch k-vectors, a fresh seeded batch drawn on
every evaluation as the reference does (Force_long.jl:235), Julia-reference
semantics -- evaluated by the FP32+FP64-fix path (short + self + long range).
The plain FP64 GPU path is timed in the same run and reported beside it, with
the FP32 path's force error against it (both on the same batch).

Multi-GPU (torchrun): one independent system per rank (seeded per rank), no
data-path collective; value = total evaluations/s over all ranks ("weak").

--workload batch measures the many-system case instead: 256 independent slabs
(N ~ U[200, 5000], density 0.01, Lz ~ U[5, 20], P = 200 each), FP32+fix,
velocity-Verlet steps (dt = 1e-3, unit masses) recorded once as a CUDA graph
and replayed --steps times; value = MD steps/s of the whole batch.

--workload exact measures the exact (non-random-batch) long range: every
lattice k with 0 < |k| < 1.0 (7,9xx vectors) weighted by exp(-k^2 / 4 alpha) on a
1e4-particle slab at the benchmark density; value = long-range evaluations/s
(FP32+fix), the FP64 path and the oracle's CPU rate beside it.

--impl reference times the FP64 CPU restatement of the reference algorithm
(oracle/, OpenMP on all host cores) on complete evaluations of the same
system, each with a fresh batch drawn the reference's way (K_set_generator
probabilities, weighted sampling with replacement); it times as many of the
requested steps as fit in about two minutes and reports that count.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "QEM force evals/s at N=1e5: FP32+FP64-fix vs FP64 GPU at ≤1e-5 force err"
UNIT = "evals/s"
FLOPS_PER_PAIR_NODE = 100   # op model per short-range quadrature node (FP32 flops)
SFU_PER_PAIR_NODE = 6       # MUFU ops per node in the same model
L2_FLUSH_BYTES = 256 << 20  # > 126 MB L2


REF_BUDGET_S = 120.0        # wall time of the reference arm's timed evaluations


def slab_config(cfg, Np):
    """The `config` of the N = 1e5 slab line: the same dict on both arms."""
    return {"workload": f"QEM slab N={cfg['N']} Lx=Ly={cfg['L'][0]:g} Lz=10 gamma=0.95/0.95 alpha=0.1 r_c=10 "
                        f"N_t=30 P={cfg['P']} (short+self+long), Julia-reference semantics",
            "N": cfg["N"], "pairs": int(Np), "P": cfg["P"],
            "kset": "a fresh seeded random batch of P k-vectors on every evaluation (Force_long.jl:235)",
            "l2": "GPU arm: L2 flushed between steps (256 MiB write outside the per-step timing)"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--N", type=int, default=100_000)
    ap.add_argument("--workload", choices=["slab", "batch", "exact"], default="slab",
                    help="slab: the N = 1e5 benchmark system (default); batch: 256 independent slabs, "
                         "graph-replayed velocity-Verlet steps; exact: the exact k-sum long range")
    return ap.parse_args()


# ----------------------------------------------------------------------------- clocks
class Clocks:
    """nvidia-smi sampler (200 ms) running across the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.rows = []
        self.proc = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "100", "-i", str(gpu_index)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t0 = time.perf_counter()
            while not self.rows and time.perf_counter() - t0 < 3.0 and self.proc.poll() is None:
                time.sleep(0.02)  # the first sample precedes the timed region
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [s.strip() for s in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ----------------------------------------------------------------------------- ranks
def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def max_over_ranks(v: float, world: int, device):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist

    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


# ----------------------------------------------------------------------------- CPU baseline
class RefEvaluator:
    """Complete FP64 evaluations of a slab by the CPU restatement of the
    reference (oracle/, OpenMP on all host cores): the neighbour list, every
    pair and self term, and the long range with a fresh batch per evaluation
    drawn as the reference draws it (K_set_generator table, weighted sampling
    with replacement, Force_long.jl:235)."""

    def __init__(self, cfg, seed=7):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import numpy as np

        import oracle as O

        self.O, self.cfg = O, cfg
        self.p = O.params(cfg["L"], cfg["alpha"], cfg["r_cutoff"], cfg["gamma_down"], cfg["gamma_up"],
                          accuracy=cfg["accuracy"], N_t=cfg["N_t"])
        self.K, Prob, self.sum_K = O.kset_generator(cfg["L"][0], cfg["L"][1], cfg["alpha"], cfg["accuracy"])
        self.Prob = Prob.astype(np.float64) / Prob.astype(np.float64).sum()
        self.rng = np.random.default_rng(seed)
        self.cores = int(O.max_threads())
        self.npairs = 0

    def __call__(self):
        O, cfg = self.O, self.cfg
        k3 = self.K[self.rng.choice(len(self.K), size=cfg["P"], replace=True, p=self.Prob)]
        pl = O.pairs(self.p, cfg["xyz"], method="cells")
        self.npairs = len(pl)
        return O.short_forces(self.p, cfg["xyz"], cfg["q"], pl) + O.F_long(self.p, cfg["xyz"], cfg["q"], k3,
                                                                          self.sum_K)

    def describe(self, n, seconds):
        c = self.cfg
        return (f"oracle FP64 on {self.cores} threads: {n} complete evaluation(s) of the N={c['N']} slab "
                f"({self.npairs} pairs, {c['N']} self terms, P={c['P']} k-vectors over all N, a fresh batch "
                f"each), {seconds:.1f} s each")


# ----------------------------------------------------------------------------- adjoint
def backward_timing(lib, local, dev, K=40):
    """qem_backward (FP64) on the differentiation workload -- config 3: N = 2e4,
    |q| ~ U[0.5, 1.5] re-neutralised, Lx = Ly = 450, Lz = 10, gamma_up = 0.8,
    gamma_down = -0.6, P = 500, loss = E + sum_i w_i . F_i with w ~ N(0, 1) --
    on device buffers, beside the FP64 forward pass with energy it
    differentiates (CUDA events, K calls each after two warm-up calls)."""
    import numpy as np
    import torch

    from qem4molly_b200 import workloads as W

    cfg = W.config3()
    e = W.engine_for(cfg, "fp64", device=local)
    x = torch.tensor(cfg["xyz"], dtype=torch.float64, device=dev)
    q = torch.tensor(cfg["q"], dtype=torch.float64, device=dev)
    w = torch.tensor(np.random.default_rng(20261206).normal(size=cfg["xyz"].shape), dtype=torch.float64, device=dev)
    gx, gq, F = torch.empty_like(x), torch.empty_like(q), torch.empty_like(x)
    stream = torch.cuda.current_stream(dev)

    def timed(fn):
        for _ in range(2):
            fn()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        for _ in range(K):
            fn()
        b.record(stream)
        b.synchronize()
        return a.elapsed_time(b) / K

    ms_b = timed(lambda: e.backward_device(x, q, w, 1.0, gx, gq))
    ms_f = timed(lambda: e.forces_device(x, q, F, energy=True))
    p64 = C.c_double(0)
    lib.qem_measure_fp64_peak(local, C.byref(p64))
    e.close()
    return {"workload": f"config 3: N={cfg['N']} Lx=Ly=450 Lz=10 gamma_up=0.8 gamma_down=-0.6 P={cfg['P']}, "
                        "loss = E + sum_i w_i . F_i, gradients w.r.t. positions, charges and both gammas (FP64)",
            "ms": ms_b, "value": 1000.0 / ms_b, "unit": "backward passes/s", "forward_fp64_energy_ms": ms_f,
            "ratio_to_forward": ms_b / ms_f, "fp64_peak_tflops": p64.value,
            "note": "device buffers; includes the neighbour list, the forward quantities the backward needs and "
                    "the short- and long-range adjoint passes"}


# ----------------------------------------------------------------------------- GPU arm
def run_ours(args):
    import numpy as np
    import torch

    from qem4molly_b200 import _lib as L
    from qem4molly_b200 import workloads as W

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    lib = L.load()
    fp32_peak, mufu_peak = C.c_double(0), C.c_double(0)
    lib.qem_measure_peaks(local, C.byref(fp32_peak), C.byref(mufu_peak))

    cfg = W.config2(N=args.N, seed=None if rank == 0 else W.SEED0 + 2 + 1000 * rank)
    # a fresh random batch on every evaluation, drawn on the device (batch n of the seed at call n)
    kseed = 7 + 1000 * rank
    e32 = W.engine_for(cfg, "fp32", mode_flags=L.QEM_RESAMPLE_KSET, seed=kseed, device=local)
    e64 = W.engine_for(cfg, "fp64", mode_flags=L.QEM_RESAMPLE_KSET, seed=kseed, device=local)
    x = torch.tensor(cfg["xyz"], dtype=torch.float64, device=dev)
    q = torch.tensor(cfg["q"], dtype=torch.float64, device=dev)
    F = torch.empty_like(x)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    terms = L.QEM_TERM_ALL

    def timed(e, K):
        per = []
        for _ in range(K):
            flush.zero_()  # evict the 126 MB L2 between steps (outside the event window)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            e.forces_device(x, q, F, terms=terms)
            b.record(stream)
            b.synchronize()
            per.append(a.elapsed_time(b))
        return per

    def kernel_times(e, K, terms=terms, min_s=0.0):
        """Per-phase CUDA-event times (on the streams each phase is launched on) over K profiled steps
        (more while under min_s seconds of wall time, so the clock sampler sees the load)."""
        e.set_profiling(True)
        kt = {}
        t0 = time.perf_counter()
        it = 0
        while it < K or time.perf_counter() - t0 < min_s:
            it += 1
            flush.zero_()
            e.forces_device(x, q, F, terms=terms)
            for k, v in e.timings().items():
                kt.setdefault(k, []).append(v)
        e.set_profiling(False)
        return {k: float(np.mean(v)) for k, v in kt.items()}

    for _ in range(max(args.warmup, 3)):
        e32.forces_device(x, q, F, terms=terms)
        e64.forces_device(x, q, F, terms=terms)
    torch.cuda.synchronize()
    barrier(world)
    clocks = Clocks(local)
    torch.cuda.synchronize()
    barrier(world)
    per32 = timed(e32, args.steps)
    torch.cuda.synchronize()
    barrier(world)
    kt32 = kernel_times(e32, args.steps, min_s=1.0)
    counts = e32.counts()  # kernels of one full evaluation (before the short-range-only pass)
    # the pair kernel alone on the GPU (short range only): in the full step the
    # high-priority long-range chain shares its SMs and stretches its span
    kt32_short = kernel_times(e32, args.steps, terms=L.QEM_TERM_SHORT)
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    ms32 = max_over_ranks(float(np.sum(per32)) / args.steps, world, dev)
    K64 = max(3, args.steps // 4)
    per64 = timed(e64, K64)
    ms64 = max_over_ranks(float(np.sum(per64)) / K64, world, dev)
    kt64 = kernel_times(e64, K64)

    # accuracy of the FP32+fix path against the plain FP64 path (parity-tested against the
    # oracle) on the same batch: both engines restart at batch 0 of the seed
    e32.sample_kset(kseed, cfg["P"])
    e64.sample_kset(kseed, cfg["P"])
    e32.forces_device(x, q, F, terms=terms)
    F32 = F.cpu().numpy().copy()
    e64.forces_device(x, q, F, terms=terms)
    F64 = F.cpu().numpy().copy()
    err, err_max = W.rel_err(F32, F64)

    # end to end through the public API with pinned host buffers (H2D + D2H inside the timed region)
    xh = torch.tensor(cfg["xyz"], dtype=torch.float64).pin_memory()
    qh = torch.tensor(cfg["q"], dtype=torch.float64).pin_memory()
    Fh = torch.empty_like(xh).pin_memory()
    for _ in range(2):
        e32.forces(xh.numpy(), qh.numpy(), terms=terms, out=Fh.numpy())
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e32.forces(xh.numpy(), qh.numpy(), terms=terms, out=Fh.numpy())
    t_e2e = max_over_ranks(time.perf_counter() - t0, world, dev)
    e2e = {"value": world * args.steps / t_e2e, "unit": UNIT, "h2d_bytes_per_step": int(xh.numel() * 8 + qh.numel() * 8),
           "d2h_bytes_per_step": int(Fh.numel() * 8)}

    backward = backward_timing(lib, local, dev)

    # roofline of the dominant kernel (short-range pair quadrature, FP32)
    Np = counts["pairs"]
    nodes = Np * 8 * cfg["N_t"]
    t_pair = kt32_short.get("short_pair", float("nan")) * 1e-3
    achieved = nodes * FLOPS_PER_PAIR_NODE / t_pair / 1e12
    traffic = None
    tf = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tf):
        traffic = json.load(open(tf)).get("short_pair_fp32_bytes_per_launch")
    roofline = {"bound": "fp32", "kernel": "k_short_pair<FP32>", "achieved": achieved, "peak": fp32_peak.value,
                "unit": "TFLOP/s", "frac": achieved / fp32_peak.value if fp32_peak.value else None,
                "traffic": traffic,
                "peak_source": "measured in this run (qem_measure_peaks: the larger of scalar and packed FP32x2 FMA chains); MEASURED_PEAKS.json has no FP32 figure",
                "work_model": f"{FLOPS_PER_PAIR_NODE} FP32 flops + {SFU_PER_PAIR_NODE} MUFU ops per pair-node; "
                              f"{Np} pairs x 8 x {cfg['N_t']} nodes per launch",
                "mufu": {"achieved": nodes * SFU_PER_PAIR_NODE / t_pair / 1e12, "peak": mufu_peak.value,
                         "unit": "Tops/s"}}

    out = {"metric": METRIC, "value": world * 1000.0 / ms32, "unit": UNIT, "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms32, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32+f64fix", "data": "synthetic (seeded, per-rank system)",
           "config": slab_config(cfg, Np),
           "notes": {"precision": "FP32+FP64-fix; the fp64 key is the plain FP64 GPU path on the same workload",
                     "kernel_times": "kernel_ms comes from a profiled pass of the same steps right after the "
                                     "timed loop (per-phase CUDA events on their own streams; the long range "
                                     "overlaps the pair kernel there); roofline.achieved uses the pair kernel's "
                                     "span in a profiled short-range-only pass (the kernel alone on the GPU); "
                                     "the timed loop itself runs the unprofiled production path",
                     "parallelism": f"{world} independent systems (one per GPU); per GPU the long range "
                                    "runs on a second stream concurrently with the short range"},
           "e2e": e2e, "gpu_launches": int(counts["launches"]) * args.steps, "roofline": roofline,
           "fp64": {"value": world * 1000.0 / ms64, "ms_per_step": ms64, "steps": K64},
           "speedup_vs_fp64": ms64 / ms32, "force_rel_err_vs_fp64": err, "force_max_err_vs_fp64_rms": err_max,
           "kernel_ms": {"fp32": kt32, "fp64": kt64, "fp32_short_only": kt32_short}, "backward": backward,
           "clocks": clk}
    if rank == 0 and world == 1:
        ref = RefEvaluator(cfg)
        t0 = time.perf_counter()
        ref()
        t_ref = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": 1.0 / t_ref, "unit": UNIT, "cores": ref.cores, "kind": "port",
                               "sample": ref.describe(1, t_ref)}
    e32.close()
    e64.close()
    if world == 1:
        # the two other workloads, recorded in this line too (each times its own steps with CUDA events)
        import argparse

        sub = argparse.Namespace(**vars(args))
        sub.steps, sub.warmup = 300, 3
        bo = run_batch(sub, quiet=True)
        out["batch_md"] = {"metric": bo["metric"], "value": bo["value"], "unit": bo["unit"],
                           "ms_per_step": bo["ms_per_step"], "steps": bo["steps"],
                           "workload": bo["config"]["workload"], "kset": bo["config"]["kset"],
                           "particles": bo["config"]["particles_per_gpu"], "batch_mode": bo["batch_mode"],
                           "batch_forces_graph_ms": bo["batch_forces_graph_ms"],
                           "particle_steps_per_s": bo["particle_steps_per_s"], "clocks": bo["clocks"]}
        sub.steps = 30
        xo = run_exact(sub, quiet=True, cpu_leg=False)
        out["exact_ksum"] = {"metric": xo["metric"], "value": xo["value"], "unit": xo["unit"],
                             "ms_per_step": xo["ms_per_step"], "steps": xo["steps"],
                             "workload": xo["config"]["workload"], "fp64_value": xo["fp64"]["value"],
                             "force_rel_err_vs_fp64": xo["force_rel_err_vs_fp64"],
                             "mufu_frac": xo["roofline"]["frac"], "clocks": xo["clocks"]}
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()



# ----------------------------------------------------------------------------- batch workload
def run_batch(args, quiet=False):
    import numpy as np
    import torch

    from qem4molly_b200 import _lib as L
    from qem4molly_b200 import workloads as W
    from qem4molly_b200.api import Batch

    rank, world, local = dist_env()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    tt = [time.perf_counter()]
    cfgs = W.config4(seed=None if rank == 0 else 20261203 + 4 + 1000 * rank)
    # a fresh random batch of k-vectors every step (Force_long.jl:235), drawn on the device
    engines = [W.engine_for(c, "fp32", mode_flags=L.QEM_RESAMPLE_KSET, seed=100 + i, device=local)
               for i, c in enumerate(cfgs)]
    tt.append(time.perf_counter())
    N = [c["N"] for c in cfgs]
    x = torch.tensor(np.concatenate([c["xyz"] for c in cfgs]), device=dev)
    q = torch.tensor(np.concatenate([c["q"] for c in cfgs]), device=dev)
    v = torch.zeros_like(x)
    F = torch.empty_like(x)
    b = Batch(engines, N)
    b.forces(x, q, F)
    tt.append(time.perf_counter())
    width, ms_eval = b.autotune(x, q, F)
    mode = b.mode()
    tt.append(time.perf_counter())
    dt = 1e-3
    b.md(max(args.warmup, 3), dt, x, v, q, F)
    tt.append(time.perf_counter())
    print("batch set-up s (systems, sizing, autotune, md warm-up):",
          [round(b_ - a_, 2) for a_, b_ in zip(tt[:-1], tt[1:])], file=sys.stderr)
    # eager reference point: one synchronous per-system evaluation of every system
    t0 = time.perf_counter()
    for c, e, o, n in zip(cfgs, engines, b.off, N):
        e.forces_device(x[o:o + n], q[o:o + n], F[o:o + n])
    torch.cuda.synchronize()
    eager_ms = 1000.0 * (time.perf_counter() - t0)
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clk = Clocks(local)
    e0.record()
    b.md(args.steps, dt, x, v, q, F)
    e1.record()
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = max_over_ranks(e0.elapsed_time(e1), world, dev)
    # the same MD with the Andersen thermostat on (kT = 1, nu = 10: p = 0.01 per step)
    K_a = max(3, min(args.steps, 200))
    b.set_thermostat(1.0, 10.0, 7)
    b.md(1, dt, x, v, q, F)  # records the thermostatted step
    torch.cuda.synchronize()
    e0.record()
    b.md(K_a, dt, x, v, q, F)
    e1.record()
    torch.cuda.synchronize()
    ms_a = max_over_ranks(e0.elapsed_time(e1), world, dev)
    barrier(world)
    if rank == 0:
        n_sys = len(cfgs) * world
        out = {"metric": "QEM velocity-Verlet steps/s, 256 independent slabs per GPU (graph-replayed)",
               "value": args.steps * 1000.0 / ms, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
               "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64fix", "data": "synthetic (seeded)",
               "config": {"workload": "256 slabs per GPU: N ~ U[200, 5000], density 0.01, Lz ~ U[5, 20], "
                                      "gamma ~ U(-0.95, 0.95)^2, alpha 0.1, r_c 10, P 200; dt 1e-3, unit masses",
                          "systems": n_sys, "particles_per_gpu": int(sum(N)),
                          "kset": "a fresh seeded random batch of P k-vectors per system on every step",
                          "l2": "working set (< 100 MB) stays in L2 between steps; not flushed"},
               "batch_mode": {"mode": mode["mode"], "pool_width": width, "ks_per_system": mode["ks"],
                              "order": ["batch", "largest first"][mode["order"]], "chunk": mode["chunk"],
                              "launches_per_evaluation": mode["launches"], "why_not_fused": mode["why"]},
               "batch_forces_graph_ms": ms_eval, "eager_per_system_forces_ms": eager_ms,
               "particle_steps_per_s": args.steps * sum(N) * world * 1000.0 / ms,
               "andersen": {"kT": 1.0, "nu": 10.0, "steps": K_a, "ms_per_step": ms_a / K_a,
                            "value": K_a * 1000.0 / ms_a, "unit": "steps/s"},
               "clocks": clocks}
        if not quiet:
            print(json.dumps(out), flush=True)
        return out
    return None

# ----------------------------------------------------------------------------- exact k-sum workload
FLOPS_PER_K_TERM = 80   # op model per (k, particle) long-range term (FP32 flops)
SFU_PER_K_TERM = 4      # MUFU ops per term in the same model


def run_exact(args, quiet=False, cpu_leg=True):
    import numpy as np
    import torch

    from qem4molly_b200 import _lib as L
    from qem4molly_b200 import workloads as W

    rank, world, local = dist_env()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    lib = L.load()
    fp32_peak, mufu_peak = C.c_double(0), C.c_double(0)
    lib.qem_measure_peaks(local, C.byref(fp32_peak), C.byref(mufu_peak))
    N, k_c = 10_000, 1.0
    cfg = W.config2(N=N, seed=None if rank == 0 else W.SEED0 + 2 + 1000 * rank)
    cfg["L"] = (1000.0 * np.sqrt(N / 100_000), 1000.0 * np.sqrt(N / 100_000), 10.0)
    rng = np.random.default_rng(W.SEED0 + 6 + 1000 * rank)
    cfg["xyz"] = np.stack([rng.random(N) * cfg["L"][0], rng.random(N) * cfg["L"][1], 0.5 + 9 * rng.random(N)], 1)
    engines = {}
    for prec in ("fp32", "fp64"):
        e = W.engine_for(cfg, prec, device=local)
        P = e.set_kset_exact(k_c)
        engines[prec] = e
    x = torch.tensor(cfg["xyz"], dtype=torch.float64, device=dev)
    q = torch.tensor(cfg["q"], dtype=torch.float64, device=dev)
    F = torch.empty_like(x)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    terms = L.QEM_TERM_LONG

    def timed(e, K):
        per = []
        for _ in range(K):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            e.forces_device(x, q, F, terms=terms)
            b.record(stream)
            b.synchronize()
            per.append(a.elapsed_time(b))
        return per

    for e in engines.values():
        for _ in range(max(args.warmup, 3)):
            e.forces_device(x, q, F, terms=terms)
    torch.cuda.synchronize()
    barrier(world)
    clk = Clocks(local)
    K = max(3, min(args.steps, 100))
    ms32 = max_over_ranks(float(np.mean(timed(engines["fp32"], K))), world, dev)
    ms64 = max_over_ranks(float(np.mean(timed(engines["fp64"], max(3, K // 4)))), world, dev)
    clocks = clk.stop()
    F32 = engines["fp32"].forces(cfg["xyz"], cfg["q"], terms=terms)
    F64 = engines["fp64"].forces(cfg["xyz"], cfg["q"], terms=terms)
    err, err_max = W.rel_err(F32, F64)
    launches = int(engines["fp32"].counts()["launches"])
    terms_pn = P * N
    out = None
    if rank == 0:
        out = {"metric": "QEM exact k-sum long-range evals/s (every lattice k with 0 < |k| < k_c, no random batch)",
               "value": world * 1000.0 / ms32, "unit": "evals/s", "n_gpus": world, "steps": K,
               "warmup": max(args.warmup, 3), "ms_per_step": ms32, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f32+f64fix", "data": "synthetic (seeded)",
               "config": {"workload": f"QEM slab N={N} Lx=Ly={cfg['L'][0]:.1f} Lz=10 gamma=0.95/0.95 alpha=0.1, "
                                      f"exact k-sum k_c={k_c} ({P} k-vectors), long range only",
                          "N": N, "P": P, "k_cutoff": k_c,
                          "l2": "flushed between steps (256 MiB write outside the per-step CUDA events)"},
               "gpu_launches": launches * K,
               "roofline": {"bound": "mufu", "work_model": f"{FLOPS_PER_K_TERM} FP32 flops + {SFU_PER_K_TERM} MUFU "
                                                          f"ops per (k, particle) term, {terms_pn} terms per evaluation",
                            "achieved": terms_pn * SFU_PER_K_TERM / (ms32 * 1e-3) / 1e12, "peak": mufu_peak.value,
                            "unit": "Tops/s",
                            "frac": terms_pn * SFU_PER_K_TERM / (ms32 * 1e-3) / 1e12 / mufu_peak.value,
                            "fp32": {"achieved": terms_pn * FLOPS_PER_K_TERM / (ms32 * 1e-3) / 1e12,
                                     "peak": fp32_peak.value, "unit": "TFLOP/s"},
                            "peak_source": "measured in this run (qem_measure_peaks)", "traffic": None},
               "fp64": {"value": world * 1000.0 / ms64, "ms_per_step": ms64},
               "force_rel_err_vs_fp64": err, "force_max_err_vs_fp64_rms": err_max, "clocks": clocks}
    if rank == 0 and world == 1 and cpu_leg:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O

        p = O.params(cfg["L"], cfg["alpha"], cfg["r_cutoff"], cfg["gamma_down"], cfg["gamma_up"])
        k3, w = O.exact_kset(cfg["L"], cfg["alpha"], k_c)
        n_s = min(P, 1000)
        t0 = time.perf_counter()
        O.F_long_weighted(p, cfg["xyz"], cfg["q"], k3[:n_s], w[:n_s])
        t_s = time.perf_counter() - t0
        cores = int(O.lib().qo_max_threads())
        out["cpu_baseline"] = {"value": 1.0 / (t_s * P / n_s), "unit": "evals/s", "cores": cores, "kind": "port",
                               "sample": f"oracle FP64 on {cores} threads: {n_s} of {P} k-vectors over all {N} "
                                         f"particles ({t_s:.1f} s), extrapolated to the full k-set"}
    if rank == 0 and not quiet:
        print(json.dumps(out), flush=True)
    return out


# ----------------------------------------------------------------------------- reference arm
def run_reference(args):
    """Complete evaluations by RefEvaluator.  One untimed warm-up evaluation
    sizes the run: as many of the requested steps as fit in REF_BUDGET_S are
    timed, and the line reports that count."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import numpy as np

    from qem4molly_b200 import workloads as W

    cfg = W.config2(N=args.N)
    ref = RefEvaluator(cfg)
    t0 = time.perf_counter()
    ref()
    t_warm = time.perf_counter() - t0
    steps = max(1, min(args.steps, int(REF_BUDGET_S / max(t_warm, 1e-3))))
    per = []
    for _ in range(steps):
        t0 = time.perf_counter()
        ref()
        per.append(time.perf_counter() - t0)
    ms = 1000.0 * float(np.mean(per))
    value = 1000.0 / ms
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": steps, "warmup": 1,
           "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (seeded)", "impl": "reference", "config": slab_config(cfg, ref.npairs),
           "requested_steps": args.steps,
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": ref.cores, "kind": "port",
                            "sample": ref.describe(steps, ms / 1000.0)},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "timed_wall_s": float(np.sum(per)), "warmup_s": t_warm}
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batch":
        run_batch(args)
    elif args.workload == "exact":
        run_exact(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
