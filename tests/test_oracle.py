"""The oracle (CPU restatement) pinned against the reference's own outputs (CPU only).

Golden fixtures in tests/golden/ were produced by the reference compiled from its sources
(tests/golden/make_golden.py); when oracle/_ref is present the oracle is also compared live.
"""
import json
import os

import numpy as np
import pytest

from oracle import rc_oracle as O
from oracle import ref_io
from rayleighchebyshevgpgpu_b200 import problems

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_cpoly_xstar_matches_reference_golden():
    g = json.load(open(os.path.join(GOLD, "cpoly.json")))
    xs = np.array([O.xstar(m) for m in range(1, 201)])
    ux = np.array([O.upper_xstar(m) for m in range(1, 201)])
    np.testing.assert_allclose(xs, g["xstar"], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(ux, g["upper_xstar"], rtol=1e-14, atol=0)


def test_cpoly_star_degree_matches_reference_golden():
    g = json.load(open(os.path.join(GOLD, "cpoly.json")))
    for q in g["queries"]:
        d, b = O.star_degree_and_bound(q["shift"], q["bound"], q["star"], q["degmax"])
        assert d == q["star_degree"]
        assert b == pytest.approx(q["star_bound"], rel=1e-10)


def test_pm_closed_form():
    # P_m(x) = sin((m+1) t)/((m+1) sin t), sin^2(t/2) = x
    for m in (2, 5, 17, 200):
        for x in (0.01, 0.2, 0.77):
            t = 2 * np.arcsin(np.sqrt(x))
            assert O.pm(m, x) == pytest.approx(np.sin((m + 1) * t) / ((m + 1) * np.sin(t)), rel=1e-9, abs=1e-12)


def test_filter_matches_reference_golden():
    g = np.load(os.path.join(GOLD, "filter_small.npz"))
    Q = problems.small_laplacian((16, 16), seed=21)
    A = O.csr_matrix(*Q.csr())
    m, bound, shift = int(g["degree"]), float(g["bound"]), float(g["shift"])
    g1, g2 = O.gammas(m, bound, shift)
    Y = O.filter_block(A, g["X"].T, m, g1, g2)
    np.testing.assert_allclose(Y.T, g["Y"], rtol=1e-12, atol=1e-12 * np.abs(g["Y"]).max())


def test_lanczos_matches_reference_golden():
    g = json.load(open(os.path.join(GOLD, "lanczos_config1.json")))
    P = problems.config1()
    A = O.csr_matrix(*P.csr())
    lz0 = np.random.default_rng(11).uniform(-1.0, 1.0, P.n)
    lmin, lmax, it = O.lanczos_bounds(A, lz0, 1e-6, "max")
    assert it == g["iters"]
    assert lmax == pytest.approx(g["lmax"], rel=1e-12)
    assert lmin == pytest.approx(g["lmin"], rel=1e-10)


def test_solve_config1_matches_reference_golden_and_lapack():
    g = json.load(open(os.path.join(GOLD, "config1_solve.json")))
    P = problems.config1()
    rp, ci, v = P.csr()
    A = O.csr_matrix(rp, ci, v)
    s = g["incr"] + g["buffer"]
    start = P.start_block(s)
    lz0 = np.random.default_rng(11).uniform(-1.0, 1.0, P.n)
    r = O.solve(A, g["k"], g["tol"], g["incr"], g["buffer"], start.T, lz0, stop=g["stop"])
    ev = r["eigenvalues"]
    np.testing.assert_allclose(ev, g["eigenvalues"], rtol=1e-10)
    np.testing.assert_allclose(ev, g["dense_eigenvalues"], rtol=1e-10)
    np.testing.assert_allclose(g["eigenvalues"], g["dense_eigenvalues"], rtol=1e-10)
    assert r["residuals"].max() <= 1e-10 * np.abs(ev).max()


def test_oracle_laplacian_1d_analytic():
    n, k = 200, 6
    Q = problems.small_laplacian((n,), seed=0, vmax=0.0)
    A = O.csr_matrix(*Q.csr())
    start = np.random.default_rng(3).standard_normal((n, 14))
    r = O.solve(A, k, 1e-10, 6, 8, start, np.random.default_rng(4).uniform(-1, 1, n))
    np.testing.assert_allclose(r["eigenvalues"], O.laplacian_1d_dirichlet(n, k), rtol=1e-10)


def test_oracle_multipass_deflation():
    # incr < k exercises found-vector deflation over several outer passes
    Q = problems.small_laplacian((20, 20), seed=5)
    A = O.csr_matrix(*Q.csr())
    start = np.random.default_rng(6).standard_normal((Q.n, 12))
    r = O.solve(A, 10, 1e-10, 4, 8, start, np.random.default_rng(7).uniform(-1, 1, Q.n))
    np.testing.assert_allclose(np.sort(r["eigenvalues"]), O.dense_lowest(A, 10), rtol=1e-9)


def test_oracle_complex_tight_binding_vs_lapack():
    Q = problems.small_laplacian((6, 6, 6), seed=9, complex_=True, flux=1.0 / 7.0)
    A = O.csr_matrix(*Q.csr())
    D = A.toarray()
    assert np.allclose(D, D.conj().T)
    rng = np.random.default_rng(10)
    start = rng.standard_normal((Q.n, 16)) + 1j * rng.standard_normal((Q.n, 16))
    r = O.solve(A, 8, 1e-10, 8, 8, start, rng.uniform(-1, 1, Q.n))
    np.testing.assert_allclose(r["eigenvalues"], O.dense_lowest(A, 8), rtol=1e-9, atol=1e-12)


@pytest.mark.skipif(not ref_io.ref_available(), reason="reference build (oracle/_ref) not present")
def test_oracle_vs_live_reference_random_problem(tmp_path):
    Q = problems.small_laplacian((24, 24), seed=31, vmax=3.0)
    rp, ci, v = Q.csr()
    A = O.csr_matrix(rp, ci, v)
    start = np.random.default_rng(32).standard_normal((16, Q.n))
    lz0 = np.random.default_rng(33).uniform(-1, 1, Q.n)
    path = str(tmp_path / "p.bin")
    ref_io.write_problem(path, rp, ci, v, start, lz0)
    ref = ref_io.run_ref("solve", path, k=8, tol=1e-10, incr=8, buffer=8, stop="RESIDUAL_ONLY")
    r = O.solve(A, 8, 1e-10, 8, 8, start.T, lz0)
    np.testing.assert_allclose(r["eigenvalues"], ref["eigenvalues"], rtol=1e-10)
    lz = ref_io.run_ref("lanczos", path, tol=1e-6, which="max")
    lmin, lmax, it = O.lanczos_bounds(A, lz0, 1e-6, "max")
    assert it == lz["iters"] and lmax == pytest.approx(lz["lmax"], rel=1e-12)
