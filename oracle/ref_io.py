"""Drivers for the reference build in oracle/_ref (TEST INFRASTRUCTURE ONLY).

write_problem() writes the binary problem file read by oracle/ref_harness.cpp; run_ref() runs
the harness and parses its JSON. Used by tests/ and by bench.py's CPU-baseline leg only.
"""
from __future__ import annotations

import json
import os
import struct
import subprocess

import numpy as np

ORACLE_DIR = os.path.dirname(os.path.abspath(__file__))
REF_BIN = os.path.join(ORACLE_DIR, "_ref", "ref_harness")
# Where the reference sources lie: RC_REFERENCE_DIR, else the mount point of this build machine.
REFERENCE_DIR = os.environ.get("RC_REFERENCE_DIR", "/root/reference")


def ref_available() -> bool:
    return os.path.exists(REF_BIN) and os.access(REF_BIN, os.X_OK)


def reference_present(reference_dir: str | None = None) -> bool:
    return os.path.isdir(reference_dir or REFERENCE_DIR)


def build_ref(reference_dir: str | None = None, targets=("_ref/ref_harness",)) -> bool:
    """Compile the reference harness (and any other oracle/Makefile targets) from the reference
    sources, when they are present."""
    reference_dir = reference_dir or REFERENCE_DIR
    if not os.path.isdir(reference_dir):
        return ref_available()
    r = subprocess.run(["make", "-C", ORACLE_DIR, f"REF={reference_dir}", *targets], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle/_ref build failed:\n{r.stdout}\n{r.stderr}")
    return ref_available()


CONTAINERS_BIN = os.path.join(ORACLE_DIR, "_ref", "lmcuda_reference_containers")


GPU_SOLVE_BIN = os.path.join(ORACLE_DIR, "_ref", "ref_gpu_solve")


def build_gpu_solve(reference_dir: str | None = None) -> bool:
    """The reference's own FP64 GPU solver on a cuSPARSE operator (oracle/ref_gpu_solve.cu)."""
    if reference_present(reference_dir):
        build_ref(reference_dir, targets=("_ref/ref_gpu_solve",))
    return os.path.exists(GPU_SOLVE_BIN)


def run_gpu_solve(problem_path: str, k: int, incr: int, buffer: int, tol: float, repeats: int = 1,
                  timeout: float = 1800) -> dict:
    """Run the reference's GPU solver on a problem file; its JSON line as a dict."""
    if not os.path.exists(GPU_SOLVE_BIN):
        raise RuntimeError("oracle/_ref/ref_gpu_solve is not built")
    cmd = [GPU_SOLVE_BIN, problem_path, str(k), str(incr), str(buffer), repr(float(tol)), str(repeats)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"ref_gpu_solve failed ({r.returncode}): {r.stderr[-2000:]}")
    return json.loads(r.stdout.strip().splitlines()[-1])


def build_containers_driver(reference_dir: str | None = None) -> bool:
    """The drop-in driver over the reference's own containers (needs the built library)."""
    if reference_present(reference_dir):
        build_ref(reference_dir, targets=("_ref/lmcuda_reference_containers",))
    return os.path.exists(CONTAINERS_BIN)


def write_problem(path: str, rowptr, colind, vals, start=None, lz0=None) -> None:
    """start: C-ordered (s, n) array (row j = column j of the block); lz0: length-n vector."""
    rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
    colind = np.ascontiguousarray(colind, dtype=np.int32)
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    n = rowptr.size - 1
    s = 0 if start is None else int(start.shape[0])
    with open(path, "wb") as f:
        f.write(b"RCPB")
        f.write(struct.pack("<i", 1))
        f.write(struct.pack("<4q", n, colind.size, s, 0 if lz0 is None else 1))
        f.write(rowptr.tobytes())
        f.write(colind.tobytes())
        f.write(vals.tobytes())
        if s:
            f.write(np.ascontiguousarray(start, dtype=np.float64).tobytes())
        if lz0 is not None:
            f.write(np.ascontiguousarray(lz0, dtype=np.float64).tobytes())


def run_ref(mode: str, problem_path: str | None = None, timeout: float = 3600, **kw) -> dict:
    if not ref_available():
        raise RuntimeError("oracle/_ref/ref_harness is not built")
    cmd = [REF_BIN, mode]
    if problem_path:
        cmd.append(problem_path)
    cmd += [f"{k}={v}" for k, v in kw.items()]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"ref_harness failed ({r.returncode}): {r.stderr}")
    return json.loads(r.stdout)
