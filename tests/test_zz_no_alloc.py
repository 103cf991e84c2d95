"""qem_long_forces_noalloc: the long-range forces for callers that cannot call
cudaMalloc (a host framework that owns all device memory in its own pool, or
a real-time loop that must not enter the CUDA allocator).  Its scratch is a
fixed array inside libqem.so, so it is checked here against the allocating
entry point (qem_long_forces through a handle) on the same system and k-set,
twice in a row, since every call reuses the same scratch.  This file is
collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

from qem4molly_b200 import _lib as L
from qem4molly_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("fp32", 1e-12)])
def test_noalloc_matches_allocating_entry_point(prec, tol):
    import torch

    cfg = W.config2(N=20_000, seed=99)
    e = W.engine_for(cfg, prec, seed=11)
    k3, sK = e.get_kset()
    F_ref = e.forces(cfg["xyz"], cfg["q"], terms=L.QEM_TERM_LONG)
    lib = L.load()
    x = torch.tensor(cfg["xyz"], dtype=torch.float64, device="cuda")
    q = torch.tensor(cfg["q"], dtype=torch.float64, device="cuda")
    k3c = np.ascontiguousarray(k3)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call in range(2):
        F = torch.full_like(x, float("nan"))
        st = lib.qem_long_forces_noalloc(C.byref(e.params), cfg["N"], C.c_void_p(x.data_ptr()),
                                         C.c_void_p(q.data_ptr()), k3c.shape[0],
                                         k3c.ctypes.data_as(C.POINTER(C.c_double)), sK, C.c_void_p(F.data_ptr()),
                                         stream)
        assert st == 0, f"call {call}: status {st}"
        assert W.rel_err(F.cpu().numpy(), F_ref)[0] <= tol, f"call {call}"


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
    kbig = np.tile(k3, (513, 1))
    assert lib.qem_long_forces_noalloc(C.byref(p), 100, C.c_void_p(x.data_ptr()), C.c_void_p(q.data_ptr()), 513,
                                       kbig.ctypes.data_as(C.POINTER(C.c_double)), 1.0, C.c_void_p(F.data_ptr()),
                                       None) == 1

