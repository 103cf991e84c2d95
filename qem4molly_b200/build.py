"""Build libqem.so in place with nvcc for sm_100a (B200).

    python -m qem4molly_b200.build          # or qem4molly_b200.build.build_lib()

The library is plain CUDA C++ behind the C-ABI of include/qem.h; it links the
CUDA runtime statically and does not depend on torch.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libqem.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + [os.path.join(ROOT, "include", "qem.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build_lib(force: bool = False, verbose: bool = False, extra=None) -> str:
    """Compiles each .cu file to an object (in parallel, under _build/) and
    links them into libqem.so; no relocatable device code is needed, since no
    kernel calls device code of another file."""
    if not force and not _stale():
        return LIB
    from concurrent.futures import ThreadPoolExecutor

    objdir = os.path.join(PKG, "_build")
    os.makedirs(objdir, exist_ok=True)
    flags = [*ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include"),
             *(extra or [])]
    jobs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.splitext(os.path.basename(src))[0] + ".o")
        jobs.append((obj, [nvcc(), *flags, "-c", src, "-o", obj]))

    def run(job):
        if verbose:
            print(" ".join(job[1]))
        return subprocess.run(job[1], capture_output=not verbose, text=True)

    with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
        results = list(ex.map(run, jobs))
    for (obj, cmd), r in zip(jobs, results):
        if r.returncode != 0:
            if r.stderr:
                sys.stderr.write(r.stderr)
            raise subprocess.CalledProcessError(r.returncode, cmd)
        if verbose is False and r.stderr and "ptxas" in r.stderr:
            sys.stderr.write(r.stderr)
    tmp = LIB + ".tmp"
    link = [nvcc(), *ARCH, "-shared", "-o", tmp, *[o for o, _ in jobs]]
    if verbose:
        print(" ".join(link))
    subprocess.run(link, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build_lib(force="--force" in sys.argv, verbose=True,
              extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else None)
    print(LIB)
