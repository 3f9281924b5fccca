"""Build librcb200.so (the sm_100a kernels + C ABI) in-tree with nvcc.

Usage: python -m rayleighchebyshevgpgpu_b200.build [-v]
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG_DIR, "csrc")
BUILD_DIR = os.path.join(PKG_DIR, "_build")
LIB_NAME = "librcb200.so"
LIB_PATH = os.path.join(PKG_DIR, LIB_NAME)

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH_FLAGS + [
    "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    "--expt-relaxed-constexpr", "-Xptxas", "-O3",
]
SOURCES = ["rc_filter.cu", "rc_filter_rm.cu", "rc_dense.cu", "rc_gemm.cu", "rc_noalloc.cu", "rc_lanczos.cu", "rc_solver.cu", "rc_capi.cu",
           "rc_batch.cu", "rc_serve.cu", "rc_resid.cu", "rc_corrapi.cu"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def build(verbose: bool = False, force: bool = False, extra_flags: list[str] | None = None) -> str:
    """Compile every CUDA source for sm_100a and link the shared library. Returns its path."""
    os.makedirs(BUILD_DIR, exist_ok=True)
    nvcc = _nvcc()
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(PKG_DIR, "..", "include", "rc_b200.h"))
    flags = NVCC_FLAGS + (extra_flags or [])
    objs = []
    jobs = []
    for src in SOURCES:
        sp = os.path.join(CSRC, src)
        obj = os.path.join(BUILD_DIR, src.replace(".cu", ".o"))
        objs.append(obj)
        if force or not _newer(obj, [sp] + headers):
            jobs.append([nvcc] + flags + ["-c", sp, "-o", obj])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose and (r.stdout or r.stderr):
            print(r.stdout, r.stderr)
        return r

    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        list(ex.map(run, jobs))
    if jobs or not os.path.exists(LIB_PATH):
        run([nvcc] + ARCH_FLAGS + ["-shared", "-o", LIB_PATH] + objs + ["-lcudart", "-lpthread"])
    return LIB_PATH


if __name__ == "__main__":
    v = "-v" in sys.argv
    print(build(verbose=v, force="-f" in sys.argv))
