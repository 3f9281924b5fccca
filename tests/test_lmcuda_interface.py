"""The templated drop-in interface include/rc_b200_lmcuda.h (the reference's RayleighChebyshevLMCuda
API over the C ABI): it compiles with a caller's own containers, and on the GPU the three operator
kinds (fused stencil, fused CSR, foreign device apply) reproduce dense LAPACK eigenvalues."""
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "lmcuda_api.cu")
PKG = os.path.join(ROOT, "rayleighchebyshevgpgpu_b200")


def _nvcc():
    return shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


def _build(tmp_path, link: bool):
    out = str(tmp_path / ("lmcuda_api" if link else "lmcuda_api.o"))
    cmd = [_nvcc(), "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-I",
           os.path.join(ROOT, "include"), SRC, "-o", out]
    if link:
        cmd += ["-L", PKG, "-lrcb200", "-Xlinker", f"-rpath={PKG}"]
    else:
        cmd.insert(1, "-c")
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


def test_interface_header_compiles(tmp_path):
    _build(tmp_path, link=False)


def _dense_lowest(k):
    nx, ny = 48, 40
    n = nx * ny
    i = np.arange(n)
    A = np.diag(4.0 + 0.5 * (1.0 + np.sin(0.7 * i)))
    for r in range(n):
        x, y = r % nx, r // nx
        for (ok, j) in ((y > 0, r - nx), (x > 0, r - 1), (x + 1 < nx, r + 1), (y + 1 < ny, r + nx)):
            if ok:
                A[r, j] = -1.0
    return np.linalg.eigvalsh(A)[:k]


@pytest.mark.gpu
def test_interface_three_operator_kinds_match_lapack(tmp_path, built_lib):
    exe = _build(tmp_path, link=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    rows = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert [d["op"] for d in rows] == ["stencil", "csr", "foreign"], r.stdout
    dense = _dense_lowest(8)
    for d in rows:
        assert d["found"] == 8 and d["cols"] == 8, d
        np.testing.assert_allclose(d["evals"], dense, rtol=1e-10)
        ev = np.asarray(d["evals"])
        assert np.max(np.asarray(d["residuals"]) / np.abs(ev)) <= 1e-10, d
        assert d["opapply"] > 0 and d["lanczos"] > 0
        assert abs(d["bounds"][0] - dense[0]) <= 1e-2 * abs(dense[0]) and d["bounds"][1] > dense[-1], d
    # the fused CSR and stencil forms of the same matrix agree to rounding
    np.testing.assert_allclose(rows[0]["evals"], rows[1]["evals"], rtol=1e-12)


def test_stop_condition_enumerators_map_to_the_c_abi(tmp_path):
    """setStopCondition's enum form: the reference's RC_Types order (DEFAULT, COMBINATION, EIGENVALUE_ONLY,
    RESIDUAL_ONLY) maps onto RC_STOP_*, DEFAULT meaning COMBINATION; a foreign enum with the same order works."""
    src = tmp_path / "stop.cpp"
    src.write_text(
        '#include <cstdio>\n#include "rc_b200_lmcuda.h"\n'
        'struct RC_Types { enum StopCondition {DEFAULT, COMBINATION, EIGENVALUE_ONLY, RESIDUAL_ONLY}; };\n'
        'int main() {\n'
        '  using R = rcb200::RC_Types;\n'
        '  std::printf("%d %d %d %d %d %d\\n", rcb200::stop_condition_value(R::DEFAULT),\n'
        '    rcb200::stop_condition_value(R::COMBINATION), rcb200::stop_condition_value(R::EIGENVALUE_ONLY),\n'
        '    rcb200::stop_condition_value(R::RESIDUAL_ONLY), rcb200::stop_condition_value(::RC_Types::RESIDUAL_ONLY),\n'
        '    RC_STOP_RESIDUAL_ONLY);\n'
        '  return 0;\n}\n')
    exe = str(tmp_path / "stop")
    gxx = shutil.which("g++") or "g++"
    r = subprocess.run([gxx, "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
                        str(src), "-o", exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([exe], capture_output=True, text=True, timeout=60).stdout.split()
    assert out == ["1", "1", "2", "3", "3", "3"]
