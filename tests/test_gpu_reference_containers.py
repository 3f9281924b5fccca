"""The drop-in interface with the reference's own containers on the GPU.

oracle/_ref/lmcuda_reference_containers (tests/cpp/lmcuda_reference_containers.cu, compiled by
oracle/Makefile from the reference's AmatrixClassLMCuda.h, AvectorClassLMCuda.h and
ArandomizeOpClassLMCuda.h) instantiates rcb200::RayleighChebyshevLMCuda with those containers, the
reference's randomize op and a cuSPARSE-backed operator with the reference's device block apply,
and solves configuration 1 (2D 5-point Laplacian 64x64 + U[0,1) potential, k = 16, tol 1e-10,
RESIDUAL_ONLY). The eigenvalues must match the reference's own CPU solve (golden fixture) to 1e-10
relative, the eigenvectors returned in the container's host mData must meet the tolerance and be
orthonormal, and the container's device copy mData_d must hold the same values."""
import json
import os
import struct
import subprocess

import numpy as np
import pytest

from oracle import ref_io
from rayleighchebyshevgpgpu_b200 import problems

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_reference_containers_solve_config1(tmp_path, built_lib):
    if not ref_io.build_containers_driver():
        pytest.skip("the driver needs the reference's headers at build time and was not built")
    g = json.load(open(os.path.join(GOLD, "config1_solve.json")))
    P = problems.config1()
    rp, ci, v = P.csr()
    path = tmp_path / "c1.bin"
    with open(path, "wb") as f:
        f.write(struct.pack("<2q", P.n, ci.size))
        f.write(np.ascontiguousarray(rp, dtype=np.int32).tobytes())
        f.write(np.ascontiguousarray(ci, dtype=np.int32).tobytes())
        f.write(np.ascontiguousarray(v, dtype=np.float64).tobytes())
    r = subprocess.run([ref_io.CONTAINERS_BIN, str(path), str(g["k"]), str(g["incr"]), str(g["buffer"]),
                        str(g["tol"])], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    d = json.loads([l for l in r.stdout.splitlines() if l.startswith("{")][-1])
    k = g["k"]
    assert d["found"] == k and d["rows"] == P.n and d["cols"] == k, d
    ev = np.asarray(d["evals"])
    np.testing.assert_allclose(ev, g["eigenvalues"], rtol=1e-10)
    rel = np.asarray(d["host_residuals"]) / np.maximum(np.abs(ev), 0.1)
    assert rel.max() <= 1.5 * g["tol"], rel.max()
    lib_rel = np.asarray(d["residuals"]) / np.maximum(np.abs(ev), 0.1)
    assert lib_rel.max() <= g["tol"] * 1.0001
    assert d["orthonormality"] < 1e-12
    assert d["device_copy_matches"] is True
    assert d["apply_calls"] > 0 and d["lanczos"] > 0
    assert d["bounds"][0] <= ev[0] * (1 + 1e-2) and d["bounds"][1] > ev[-1]
