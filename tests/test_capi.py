"""C ABI checks that need no GPU: the library loads, exports every declared symbol, and its
host-side polynomial design matches the reference's (golden fixtures) and the oracle."""
import ctypes
import json
import os
import re

import numpy as np
import pytest

from oracle import rc_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")


def _declared_symbols():
    txt = open(os.path.join(ROOT, "include", "rc_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = set(re.findall(r"\b(rc_[a-z0-9_]+)\s*\(", txt))
    return sorted(n for n in names if not n.endswith("_fn"))


def test_library_exports_every_declared_symbol(built_lib):
    lib = ctypes.CDLL(built_lib)
    syms = _declared_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_covers_header(built_lib):
    from rayleighchebyshevgpgpu_b200 import _capi
    assert set(_declared_symbols()) <= set(_capi.SIGNATURES)
    _capi.lib()
    assert _capi.lib().rc_abi_version() == 1


def test_struct_layouts_match_header(built_lib):
    # sizeof(rc_solve_params) / sizeof(rc_solve_info) computed by a C compile of the header
    import subprocess
    import tempfile
    src = ('#include "rc_b200.h"\n#include <stdio.h>\n#include <stddef.h>\nint main(){printf("%zu %zu %zu %zu",'
           'sizeof(rc_solve_params), sizeof(rc_solve_info), offsetof(rc_solve_params, randomize_fn),'
           'offsetof(rc_solve_info, guard_value));return 0;}\n')
    d = tempfile.mkdtemp()
    with open(os.path.join(d, "t.c"), "w") as f:
        f.write(src)
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), os.path.join(d, "t.c"), "-o",
                           os.path.join(d, "t")])
    out = subprocess.check_output([os.path.join(d, "t")]).decode().split()
    from rayleighchebyshevgpgpu_b200 import _capi
    assert int(out[0]) == ctypes.sizeof(_capi.SolveParams)
    assert int(out[1]) == ctypes.sizeof(_capi.SolveInfo)
    assert int(out[2]) == _capi.SolveParams.randomize_fn.offset
    assert int(out[3]) == _capi.SolveInfo.guard_value.offset


def test_server_struct_layouts_match_header(built_lib):
    import subprocess
    import tempfile
    src = ('#include "rc_b200.h"\n#include <stdio.h>\n#include <stddef.h>\nint main(){printf("%zu %zu %zu %zu %zu",'
           'sizeof(rc_server_params), sizeof(rc_request_info), sizeof(rc_server_stats),'
           'offsetof(rc_server_params, starvation_ms), offsetof(rc_request_info, device_bytes));return 0;}\n')
    d = tempfile.mkdtemp()
    with open(os.path.join(d, "t.c"), "w") as f:
        f.write(src)
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), os.path.join(d, "t.c"), "-o",
                           os.path.join(d, "t")])
    out = [int(x) for x in subprocess.check_output([os.path.join(d, "t")]).decode().split()]
    from rayleighchebyshevgpgpu_b200 import _capi
    assert out[0] == ctypes.sizeof(_capi.ServerParams)
    assert out[1] == ctypes.sizeof(_capi.RequestInfo)
    assert out[2] == ctypes.sizeof(_capi.ServerStats)
    assert out[3] == _capi.ServerParams.starvation_ms.offset
    assert out[4] == _capi.RequestInfo.device_bytes.offset


def test_correction_job_layout_matches_header(built_lib):
    import subprocess
    import tempfile
    src = ('#include "rc_b200.h"\n#include <stdio.h>\n#include <stddef.h>\nint main(){printf("%zu %zu %zu",'
           'sizeof(rc_correction_job), offsetof(rc_correction_job, lam), offsetof(rc_correction_job, gamma2));'
           'return 0;}\n')
    d = tempfile.mkdtemp()
    with open(os.path.join(d, "t.c"), "w") as f:
        f.write(src)
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), os.path.join(d, "t.c"), "-o",
                           os.path.join(d, "t")])
    out = [int(x) for x in subprocess.check_output([os.path.join(d, "t")]).decode().split()]
    from rayleighchebyshevgpgpu_b200 import _capi
    assert out[0] == ctypes.sizeof(_capi.CorrectionJob)
    assert out[1] == _capi.CorrectionJob.lam.offset
    assert out[2] == _capi.CorrectionJob.gamma2.offset


def test_server_calls_without_a_server_return_status(built_lib):
    from rayleighchebyshevgpgpu_b200 import _capi
    L = _capi.lib()
    p = _capi.ServerParams()
    L.rc_server_params_default(ctypes.byref(p))
    assert p.max_active == 16 and p.use_graphs == 1 and p.struct_size == ctypes.sizeof(p)
    assert L.rc_server_create(None, None) == 1
    rid = ctypes.c_int64()
    assert L.rc_serve_submit(None, None, None, None, None, None, None, ctypes.byref(rid)) == 1
    assert L.rc_serve_poll(None, 1, None) == 1
    assert L.rc_serve_cancel(None, 1) == 1
    assert L.rc_server_destroy(None) == 0
    bad = _capi.ServerParams()
    L.rc_server_params_default(ctypes.byref(bad))
    bad.max_active = 0
    h = ctypes.c_void_p()
    assert L.rc_server_create(ctypes.byref(bad), ctypes.byref(h)) == 1 and not h


def test_serve_stream_matches_its_specification():
    """Configuration 4's request stream: 256 requests, n log-uniform in [1e4, 2e6], k in
    {8, 16, 32, 64}, tol in {1e-8, 1e-10}, W in [1, 8), and reproducible from its seed."""
    from rayleighchebyshevgpgpu_b200 import problems
    S = problems.serve_stream()
    T = problems.serve_stream()
    assert len(S) == 256
    ns = np.array([r.problem.n for r in S])
    assert ns.min() >= 0.95e4 and ns.max() <= 2.05e6
    assert {r.problem.k for r in S} == {8, 16, 32, 64}
    assert {r.problem.tol for r in S} == {1e-8, 1e-10}
    assert {r.problem.kind for r in S} == {5, 7}
    for a, b in zip(S[:5], T[:5]):
        assert a.problem.dims == b.problem.dims and np.array_equal(a.problem.diag, b.problem.diag)
        W = a.problem.meta["W"]
        d0 = 4.0 if a.problem.kind == 5 else 6.0
        assert 1.0 <= W < 8.0 and a.problem.diag.min() >= d0 and a.problem.diag.max() < d0 + W
    # log-uniform: about half the requests below the geometric midpoint
    mid = np.sqrt(1e4 * 2e6)
    assert 0.35 < np.mean(ns < mid) < 0.65


def test_cpoly_xstar_matches_reference_golden(built_lib):
    from rayleighchebyshevgpgpu_b200 import runtime as R
    g = json.load(open(os.path.join(GOLD, "cpoly.json")))
    xs = np.array([R.cpoly_xstar(m)[0] for m in range(1, 201)])
    ux = np.array([R.cpoly_xstar(m)[1] for m in range(1, 201)])
    np.testing.assert_allclose(xs, g["xstar"], rtol=1e-11, atol=1e-15)
    np.testing.assert_allclose(ux, g["upper_xstar"], rtol=1e-14)


def test_cpoly_star_degree_matches_reference_golden(built_lib):
    from rayleighchebyshevgpgpu_b200 import runtime as R
    g = json.load(open(os.path.join(GOLD, "cpoly.json")))
    for q in g["queries"]:
        d, b = R.cpoly_star_degree(q["shift"], q["bound"], q["star"], q["degmax"])
        assert d == q["star_degree"]
        assert b == pytest.approx(q["star_bound"], rel=1e-10)


def test_cpoly_star_degree_matches_oracle_random(built_lib):
    from rayleighchebyshevgpgpu_b200 import runtime as R
    rng = np.random.default_rng(0)
    for _ in range(200):
        lmin = rng.uniform(-3, 2)
        lmax = lmin + rng.uniform(0.5, 30)
        ls = lmin + rng.uniform(1e-3, 0.6) * (lmax - lmin)
        dm = int(rng.integers(5, 260))
        a = R.cpoly_star_degree(-lmin, lmax, ls, dm)
        b = O.star_degree_and_bound(-lmin, lmax, ls, dm)
        assert a[0] == b[0]
        assert a[1] == pytest.approx(b[1], rel=1e-9)


def test_cpoly_gammas_and_pm(built_lib):
    from rayleighchebyshevgpgpu_b200 import _capi
    from rayleighchebyshevgpgpu_b200 import runtime as R
    for m in (1, 2, 3, 50, 200):
        g = R.cpoly_gammas(m, 7.5, -0.25)
        o = O.gammas(m, 7.5, -0.25)
        assert g == pytest.approx(o, rel=1e-13)
        for x in (-0.01, 0.0, 0.3, 0.9):
            assert _capi.lib().rc_cpoly_pm(m, x) == pytest.approx(O.pm(m, x), rel=1e-12, abs=1e-14)


def test_invalid_arguments_return_status_not_exit(built_lib):
    from rayleighchebyshevgpgpu_b200 import _capi
    L = _capi.lib()
    assert L.rc_cpoly_xstar(-1, None, None) == 1  # RC_ERR_INVALID
    assert L.rc_ctx_create(0, None) != 0
    assert L.rc_solve(None, None, None, None, None, None, None, None) != 0
    assert L.rc_op_destroy(None) == 0
    assert L.rc_ctx_destroy(None) == 0


def test_problem_generators_hermitian_and_sizes():
    from rayleighchebyshevgpgpu_b200 import problems
    P = problems.config1()
    rp, ci, v = P.csr()
    assert P.n == 4096 and rp[-1] == 20224
    A = O.csr_matrix(rp, ci, v)
    assert abs(A - A.T).max() == 0
    Q = problems.small_laplacian((5, 6, 7), seed=1, complex_=True, flux=1 / 17)
    B = O.csr_matrix(*Q.csr()).toarray()
    assert np.allclose(B, B.conj().T)
    # nnz of the 7-point 128^3 operator of configuration 2: n*7 - 6*128^2
    assert 128 ** 3 * 7 - 6 * 128 ** 2 == 14581760
    assert problems.block_sizes(64) == (64, 32) and problems.block_sizes(16) == (16, 8)


def test_matrix_market_reader_symmetric_hermitian_general(tmp_path):
    """Operator ingestion: Matrix Market coordinate files become the CSR arrays of rc_op_csr_create."""
    from rayleighchebyshevgpgpu_b200.runtime import read_matrix_market
    rng = np.random.default_rng(0)
    n = 7
    B = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    for field, symm, M in (("real", "symmetric", (B + B.T).real),
                           ("complex", "hermitian", B + B.conj().T),
                           ("real", "general", (B + B.T).real)):
        M = M * (np.abs(M) > 0.8)  # sparse pattern
        np.fill_diagonal(M, np.diag(M) + 5.0)
        entries = [(r, c, M[r, c]) for r in range(n) for c in range(n)
                   if M[r, c] != 0 and (symm == "general" or r >= c)]
        path = tmp_path / f"{symm}.mtx"
        with open(path, "w") as f:
            f.write(f"%%MatrixMarket matrix coordinate {field} {symm}\n% test\n{n} {n} {len(entries)}\n")
            for r, c, v in entries:
                if field == "complex":
                    f.write(f"{r + 1} {c + 1} {float(v.real)!r} {float(v.imag)!r}\n")
                else:
                    f.write(f"{r + 1} {c + 1} {float(v.real)!r}\n")
        rp, ci, vals = read_matrix_market(str(path))
        D = np.zeros((n, n), dtype=vals.dtype)
        for r in range(n):
            for k in range(rp[r], rp[r + 1]):
                D[r, ci[k]] = vals[k]
            assert np.all(np.diff(ci[rp[r]:rp[r + 1]]) > 0)
        np.testing.assert_array_equal(D, M if field == "complex" else M.real)
