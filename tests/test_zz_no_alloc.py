"""qem_long_forces_noalloc: the long-range forces for callers that cannot call
cudaMalloc (a host framework that owns all device memory in its own pool, or
a real-time loop that must not enter the CUDA allocator).  Its scratch is a
fixed array inside libqem.so, so it is checked here against the allocating
entry point (qem_long_forces through a handle) on the same system and k-set,
twice in a row, since every call reuses the same scratch; the sizes cover the
one-block preparation path (N <= 8192), the multi-kernel path, the largest
accepted N and P, and an empty k-set.  The device's free memory must not
change across the two calls.  This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

from qem4molly_b200 import _lib as L
from qem4molly_b200 import workloads as W

pytestmark = pytest.mark.gpu

CASES = [(3000, None), (20_000, None), (20_000, 0), (L.QEM_NOALLOC_MAX_N, L.QEM_NOALLOC_MAX_P)]


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("N,P", CASES)
def test_noalloc_matches_allocating_entry_point(N, P, prec):
    import torch

    cfg = W.config2(N=N, seed=99)
    if P is not None:
        cfg["P"] = P
    e = W.engine_for(cfg, prec, seed=11)
    k3, sK = e.get_kset()
    assert k3.shape[0] == cfg["P"]
    F_ref = e.forces(cfg["xyz"], cfg["q"], terms=L.QEM_TERM_LONG)
    lib = L.load()
    x = torch.tensor(cfg["xyz"], dtype=torch.float64, device="cuda")
    q = torch.tensor(cfg["q"], dtype=torch.float64, device="cuda")
    k3c = np.ascontiguousarray(k3.reshape(-1, 3)) if k3.size else np.zeros((1, 3))
    kp = k3c.ctypes.data_as(C.POINTER(C.c_double))
    Fs = [torch.full_like(x, float("nan")) for _ in range(3)]
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def call(F):
        return lib.qem_long_forces_noalloc(C.byref(e.params), N, C.c_void_p(x.data_ptr()), C.c_void_p(q.data_ptr()),
                                           cfg["P"], kp, sK, C.c_void_p(F.data_ptr()), stream)

    assert call(Fs[0]) == 0  # warm-up: loads the kernels of this precision
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for i in (1, 2):
        st = call(Fs[i])
        assert st == 0, f"call {i}: status {st}"
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0, "device free memory changed across the calls"
    for i in (1, 2):
        assert W.rel_err(Fs[i].cpu().numpy(), F_ref)[0] <= 1e-12, f"call {i}"
    e.close()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch

    lib = L.load()
    p = L.default_params()
    p.Lx, p.Ly, p.Lz, p.alpha, p.r_cutoff = 100.0, 100.0, 10.0, 0.1, 10.0
    N = L.QEM_NOALLOC_MAX_N + 1
    x = torch.zeros((N, 3), dtype=torch.float64, device="cuda")
    q = torch.zeros(N, dtype=torch.float64, device="cuda")
    F = torch.zeros_like(x)
    k3 = np.array([[0.1, 0.0, 0.1]])
    dp = k3.ctypes.data_as(C.POINTER(C.c_double))
    assert lib.qem_long_forces_noalloc(C.byref(p), N, C.c_void_p(x.data_ptr()), C.c_void_p(q.data_ptr()), 1, dp,
                                       1.0, C.c_void_p(F.data_ptr()), None) == 1
    kbig = np.tile(k3, (L.QEM_NOALLOC_MAX_P + 1, 1))
    assert lib.qem_long_forces_noalloc(C.byref(p), 100, C.c_void_p(x.data_ptr()), C.c_void_p(q.data_ptr()),
                                       L.QEM_NOALLOC_MAX_P + 1, kbig.ctypes.data_as(C.POINTER(C.c_double)), 1.0,
                                       C.c_void_p(F.data_ptr()), None) == 1


def test_noalloc_fp32_flags_particles_far_outside_the_slab():
    """In FP32 a particle with max(k) |z - L_z/2| > 60 would overflow
    e^{+-k (z - L_z/2)}: the call reports QEM_ERR_RANGE instead of returning
    non-finite forces (FP64 evaluates it)."""
    import torch

    cfg = W.config2(N=2000, seed=5)
    e32 = W.engine_for(cfg, "fp32", seed=3)
    k3, sK = e32.get_kset()
    kmax = float(k3[:, 2].max())
    xyz = cfg["xyz"].copy()
    xyz[7, 2] = cfg["L"][2] / 2 + 61.0 / kmax
    lib = L.load()
    x = torch.tensor(xyz, dtype=torch.float64, device="cuda")
    q = torch.tensor(cfg["q"], dtype=torch.float64, device="cuda")
    F = torch.zeros_like(x)
    kp = np.ascontiguousarray(k3).ctypes.data_as(C.POINTER(C.c_double))
    st = lib.qem_long_forces_noalloc(C.byref(e32.params), cfg["N"], C.c_void_p(x.data_ptr()),
                                     C.c_void_p(q.data_ptr()), k3.shape[0], kp, sK, C.c_void_p(F.data_ptr()), None)
    assert st == 8
    e64 = W.engine_for(cfg, "fp64", seed=3)
    st = lib.qem_long_forces_noalloc(C.byref(e64.params), cfg["N"], C.c_void_p(x.data_ptr()),
                                     C.c_void_p(q.data_ptr()), k3.shape[0], kp, sK, C.c_void_p(F.data_ptr()), None)
    assert st == 0 and torch.isfinite(F).all()
    e32.close()
    e64.close()
