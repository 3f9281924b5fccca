"""Kernel-level parity on the GPU through the C ABI, against the oracle and the reference's
golden outputs. Blocks are column-major n x s, held as C-ordered (s, n) torch tensors."""
import json
import os

import numpy as np
import pytest

from oracle import rc_oracle as O
from rayleighchebyshevgpgpu_b200 import problems
from rayleighchebyshevgpgpu_b200 import runtime as R

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _host(t):
    return t.cpu().numpy()


def _ops(ctx, Q):
    return R.operator_from_problem(ctx, Q, "csr"), R.operator_from_problem(ctx, Q, "stencil")


@pytest.mark.parametrize("complex_", [False, True])
def test_spmm_matches_scipy(ctx, complex_):
    Q = problems.small_laplacian((9, 8, 7), seed=3, complex_=complex_, flux=0.13)
    A = O.csr_matrix(*Q.csr())
    rng = np.random.default_rng(1)
    s = 5
    X = rng.standard_normal((s, Q.n))
    Y = rng.standard_normal((s, Q.n))
    if complex_:
        X = X + 1j * rng.standard_normal((s, Q.n))
        Y = Y + 1j * rng.standard_normal((s, Q.n))
    alpha, beta = (0.7 - 0.2j, -1.3 + 0.5j) if complex_ else (0.7, -1.3)
    for op in _ops(ctx, Q):
        Xd, Yd = _dev(X), _dev(Y)
        R.spmm(ctx, op, Xd, Yd, s, alpha, beta)
        ctx.synchronize()
        ref = (alpha * (A @ X.T) + beta * Y.T).T
        np.testing.assert_allclose(_host(Yd), ref, rtol=1e-13, atol=1e-12)


@pytest.mark.parametrize("kind,dims", [(5, (17, 13)), (7, (11, 9, 6)), (27, (10, 9, 8))])
def test_stencil_equals_csr(ctx, kind, dims):
    n = int(np.prod(dims))
    diag = 2.0 + np.random.default_rng(kind).uniform(0, 1, n)
    Q = problems.Problem("t", dims, kind, diag, -1.0 / 26.0 if kind == 27 else -1.0)
    A = O.csr_matrix(*Q.csr())
    X = np.random.default_rng(2).standard_normal((3, n))
    for op in _ops(ctx, Q):
        Xd = _dev(X)
        Yd = _dev(np.zeros_like(X))
        R.spmm(ctx, op, Xd, Yd, 3, 1.0, 0.0)
        ctx.synchronize()
        np.testing.assert_allclose(_host(Yd), (A @ X.T).T, rtol=1e-13, atol=1e-13)


def test_filter_fp64_matches_reference_golden(ctx):
    g = np.load(os.path.join(GOLD, "filter_small.npz"))
    Q = problems.small_laplacian((16, 16), seed=21)
    m, bound, shift = int(g["degree"]), float(g["bound"]), float(g["shift"])
    g1, g2 = O.gammas(m, bound, shift)
    for op in _ops(ctx, Q):
        Xd = _dev(g["X"])
        R.filter_block(ctx, op, Xd, 3, m, g1, g2, "fp64")
        ctx.synchronize()
        np.testing.assert_allclose(_host(Xd), g["Y"], rtol=1e-11, atol=1e-12 * np.abs(g["Y"]).max())


@pytest.mark.parametrize("degree", [1, 2, 3, 8, 41])
@pytest.mark.parametrize("complex_", [False, True])
def test_filter_fp64_and_mixed_vs_oracle(ctx, degree, complex_):
    Q = problems.small_laplacian((12, 11, 10), seed=4, complex_=complex_, flux=1 / 17)
    A = O.csr_matrix(*Q.csr())
    rng = np.random.default_rng(5)
    s = 7
    X = rng.standard_normal((s, Q.n))
    if complex_:
        X = X + 1j * rng.standard_normal((s, Q.n))
    lmin = -2.0 if complex_ else 1.0
    g1, g2 = O.gammas(degree, 8.5, -lmin)
    ref = O.filter_block(A, X.T, degree, g1, g2).T
    scale = np.abs(ref).max()
    for op in _ops(ctx, Q):
        for prec, tol in (("fp64", 1e-12), ("mixed", 2e-5 * max(1, degree / 8))):
            Xd = _dev(X)
            R.filter_block(ctx, op, Xd, s, degree, g1, g2, prec)
            ctx.synchronize()
            err = np.abs(_host(Xd) - ref).max() / scale
            assert err < tol, (prec, err)


@pytest.mark.parametrize("kind,dims,s", [(27, (9, 8, 7), 12), (5, (23, 19), 6), (7, (6, 7, 9), 5)])
@pytest.mark.parametrize("degree", [2, 9])
def test_filter_stencil_kinds_vs_oracle(ctx, kind, dims, s, degree):
    n = int(np.prod(dims))
    diag = 1.0 + np.random.default_rng(kind).uniform(0, 2, n)
    Q = problems.Problem("t", dims, kind, diag, -1.0 / 26.0 if kind == 27 else -1.0)
    A = O.csr_matrix(*Q.csr())
    X = np.random.default_rng(3).standard_normal((s, n))
    g1, g2 = O.gammas(degree, 9.0, -0.5)
    ref = O.filter_block(A, X.T, degree, g1, g2).T
    for op in _ops(ctx, Q):
        for prec, tol in (("fp64", 1e-12), ("mixed", 1e-5)):
            Xd = _dev(X)
            R.filter_block(ctx, op, Xd, s, degree, g1, g2, prec)
            ctx.synchronize()
            assert np.abs(_host(Xd) - ref).max() / np.abs(ref).max() < tol


def test_cholqr_orthonormal_and_same_span(ctx):
    rng = np.random.default_rng(7)
    n, s = 5000, 40
    # columns with widely different scales and a near-dependence
    V = rng.standard_normal((n, s)) * np.logspace(0, 8, s)
    V[:, 5] = V[:, 4] * 1e3 + 1e-6 * rng.standard_normal(n)
    for complex_ in (False, True):
        X = V + (1j * rng.standard_normal((n, s)) if complex_ else 0)
        Xd = _dev(X.T)
        passes = R.cholqr(ctx, Xd, n, s, complex_)
        Qm = _host(Xd).T
        assert passes >= 2
        assert np.abs(Qm.conj().T @ Qm - np.eye(s)).max() < 1e-12
        # span: every original column lies in span(Q)
        resid = X - Qm @ (Qm.conj().T @ X)
        assert (np.linalg.norm(resid, axis=0) / np.linalg.norm(X, axis=0)).max() < 1e-6


@pytest.mark.parametrize("s", [96, 70, 33, 17])
def test_cholqr_block_widths(ctx, s):
    """Tall-skinny Gram / X*T paths at the widths of the benchmark blocks (24, 48, 96) and ragged ones."""
    rng = np.random.default_rng(s)
    n = 20011
    V = rng.standard_normal((n, s)) * np.logspace(0, 3, s)
    Xd = _dev(V.T)
    R.cholqr(ctx, Xd, n, s, False)
    Qm = _host(Xd).T
    assert np.abs(Qm.T @ Qm - np.eye(s)).max() < 1e-12
    resid = V - Qm @ (Qm.T @ V)
    assert (np.linalg.norm(resid, axis=0) / np.linalg.norm(V, axis=0)).max() < 1e-10


@pytest.mark.parametrize("s,complex_", [(24, False), (96, False), (150, False), (40, True), (130, True), (7, False),
                                        (192, True), (255, True), (256, False)])
def test_small_eigh_matches_lapack(ctx, s, complex_):
    """One-CTA Jacobi in shared memory (real s <= 118, complex s <= 82) and the grid form with the
    working copies in global memory (the wider cases)."""
    rng = np.random.default_rng(s)
    H = rng.standard_normal((s, s))
    if complex_:
        H = H + 1j * rng.standard_normal((s, s))
    H = H + H.conj().T
    H[0, 0] += 1e3  # spread
    ev, Qm = R.small_eigh(ctx, H)
    ref = np.linalg.eigvalsh(H)
    nrm = np.abs(ref).max()
    assert np.abs(ev - ref).max() < 1e-13 * nrm * s
    assert np.abs(Qm.conj().T @ Qm - np.eye(s)).max() < 1e-12 * s
    assert np.abs(H @ Qm - Qm * ev).max() < 1e-12 * nrm * s


def test_small_eigh_degenerate_cluster(ctx):
    rng = np.random.default_rng(1)
    s = 64
    U, _ = np.linalg.qr(rng.standard_normal((s, s)))
    d = np.concatenate([np.full(10, 1.0), np.full(10, 1.0 + 1e-13), np.linspace(2, 3, s - 20)])
    H = (U * d) @ U.T
    H = 0.5 * (H + H.T)
    ev, Qm = R.small_eigh(ctx, H)
    np.testing.assert_allclose(ev, np.sort(d), atol=1e-13)
    assert np.abs(Qm.T @ Qm - np.eye(s)).max() < 1e-12


@pytest.mark.parametrize("complex_", [False, True])
def test_grid_jacobi_matches_one_cta_kernel(complex_):
    """The grid Jacobi (32 CTAs, cooperative launch) and the one-CTA kernel on the same global-memory
    working copies (RCB200_JACOBI_CTAS=1) apply the same rotations: the eigenvalues agree to
    rounding and both match LAPACK on a matrix with a degenerate cluster."""
    s = 160 if complex_ else 200
    rng = np.random.default_rng(17)
    X = rng.standard_normal((s, s)) + (1j * rng.standard_normal((s, s)) if complex_ else 0)
    U, _ = np.linalg.qr(X)
    d = np.concatenate([np.full(12, 1.0), np.full(12, 1.0 + 1e-13), np.linspace(2, 5, s - 24)])
    H = (U * d) @ U.conj().T
    H = 0.5 * (H + H.conj().T)
    out = []
    for ctas in ("0", "1"):
        old = os.environ.get("RCB200_JACOBI_CTAS")
        os.environ["RCB200_JACOBI_CTAS"] = ctas
        try:
            c = R.Context(0)
        finally:
            if old is None:
                os.environ.pop("RCB200_JACOBI_CTAS", None)
            else:
                os.environ["RCB200_JACOBI_CTAS"] = old
        ev, Qm = R.small_eigh(c, H)
        c.close()
        np.testing.assert_allclose(ev, np.sort(d), atol=1e-13)
        assert np.abs(Qm.conj().T @ Qm - np.eye(s)).max() < 1e-12
        assert np.abs(H @ Qm - Qm * ev).max() < 1e-12 * s
        out.append(ev)
    np.testing.assert_allclose(out[0], out[1], atol=1e-14)


@pytest.mark.parametrize("s,complex_", [(200, False), (128, True)])
def test_grid_jacobi_is_repeatable(ctx, s, complex_):
    """The grid Jacobi's CTAs leave each barrier at different times; a round reads one copy of A and
    writes the other, so no CTA's angles can see another CTA's updates of the same round. Repeated
    calls on the same matrix must then give bitwise the same eigenvalues and vectors."""
    rng = np.random.default_rng(s + 3)
    H = rng.standard_normal((s, s)) + (1j * rng.standard_normal((s, s)) if complex_ else 0)
    H = H + H.conj().T
    ev0, Q0 = R.small_eigh(ctx, H)
    ref = np.linalg.eigvalsh(H)
    assert np.abs(ev0 - ref).max() < 1e-13 * np.abs(ref).max() * s
    for _ in range(40):
        ev, Qm = R.small_eigh(ctx, H)
        assert np.array_equal(ev, ev0)
        assert np.array_equal(Qm, Q0)


def test_small_eigh_sweep_counter(ctx):
    """rc_ctx_counter("jacobi_sweeps") reports the sweeps of the last call: a diagonal matrix needs
    none, a random one several."""
    s = 40
    R.small_eigh(ctx, np.diag(np.arange(1.0, s + 1.0)))
    assert ctx.counter("jacobi_sweeps") == 0
    rng = np.random.default_rng(5)
    H = rng.standard_normal((s, s))
    R.small_eigh(ctx, H + H.T)
    assert 3 <= ctx.counter("jacobi_sweeps") <= 20


def test_rayleigh_ritz_matches_dense(ctx):
    Q = problems.small_laplacian((14, 13, 12), seed=8)
    A = O.csr_matrix(*Q.csr())
    s = 20
    V, _ = np.linalg.qr(np.random.default_rng(9).standard_normal((Q.n, s)))
    op = R.operator_from_problem(ctx, Q, "csr")
    Vd = _dev(V.T)
    Wd = _dev(np.zeros((s, Q.n)))
    ev, res, Qm = R.rayleigh_ritz(ctx, op, Vd, Wd, s, s)
    H = V.T @ (A @ V)
    ref_ev, ref_Q = np.linalg.eigh(0.5 * (H + H.T))
    np.testing.assert_allclose(ev, ref_ev, rtol=1e-12, atol=1e-12)
    Vn = _host(Vd).T
    Wn = _host(Wd).T
    np.testing.assert_allclose(Wn, A @ Vn, atol=1e-11)
    np.testing.assert_allclose(res, np.linalg.norm(A @ Vn - Vn * ev, axis=0), rtol=1e-8, atol=1e-12)


def _ctx_with(env):
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        return R.Context(0)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


@pytest.mark.parametrize("s", [17, 40, 96, 150, 192])
def test_complex_cholqr_block_widths(ctx, s):
    """Complex Gram G = X^H X on the FP64 tensor pipe (the real view with the pair swap J for the
    imaginary part), at ragged widths and an odd row count: CholeskyQR2 gives an orthonormal basis of
    the same span."""
    rng = np.random.default_rng(s + 100)
    n = 20011
    V = (rng.standard_normal((n, s)) + 1j * rng.standard_normal((n, s))) * np.logspace(0, 3, s)
    Xd = _dev(V.T)
    R.cholqr(ctx, Xd, n, s, True)
    Qm = _host(Xd).T
    assert np.abs(Qm.conj().T @ Qm - np.eye(s)).max() < 1e-12
    resid = V - Qm @ (Qm.conj().T @ V)
    assert (np.linalg.norm(resid, axis=0) / np.linalg.norm(V, axis=0)).max() < 1e-10


@pytest.mark.parametrize("s", [40, 150, 192])
def test_complex_rayleigh_ritz_tensor_pipe_matches_dense_and_simt(ctx, s):
    """H = V^H (A V) for a complex Hermitian operator through rc_rayleigh_ritz: the tensor-pipe Gram
    gives the eigenvalues of the dense projection, and agrees with the FP64 SIMT Gram
    (RCB200_GRAM_C=0) to rounding."""
    Q = problems.small_laplacian((24, 23, 22), seed=s, complex_=True, flux=1 / 17)
    A = O.csr_matrix(*Q.csr())
    rng = np.random.default_rng(s)
    V, _ = np.linalg.qr(rng.standard_normal((Q.n, s)) + 1j * rng.standard_normal((Q.n, s)))
    H = V.conj().T @ (A @ V)
    ref_ev = np.linalg.eigvalsh(0.5 * (H + H.conj().T))
    out = []
    for c in (ctx, _ctx_with({"RCB200_GRAM_C": "0"})):
        op = R.operator_from_problem(c, Q, "csr")
        Vd = _dev(V.T)
        Wd = _dev(np.zeros((s, Q.n), dtype=np.complex128))
        ev, res, _ = R.rayleigh_ritz(c, op, Vd, Wd, s, s)
        np.testing.assert_allclose(ev, ref_ev, rtol=1e-12, atol=1e-12)
        out.append(ev)
        op.close()
        if c is not ctx:
            c.close()
    np.testing.assert_allclose(out[0], out[1], rtol=1e-13, atol=1e-13)


def test_lanczos_bounds_vs_reference_golden(ctx):
    g = json.load(open(os.path.join(GOLD, "lanczos_config1.json")))
    P = problems.config1()
    lz0 = np.random.default_rng(11).uniform(-1.0, 1.0, P.n)
    for form in ("csr", "stencil"):
        op = R.operator_from_problem(ctx, P, form)
        lmin, lmax, it = R.lanczos_bounds(ctx, op, lz0, tol=1e-6, which="max")
        assert abs(it - g["iters"]) <= 5
        assert lmax == pytest.approx(g["lmax"], rel=1e-8)
        assert lmin == pytest.approx(g["lmin"], rel=1e-5)


def test_lanczos_both_extremes_complex(ctx):
    Q = problems.small_laplacian((8, 8, 8), seed=12, complex_=True, flux=1 / 17)
    A = O.csr_matrix(*Q.csr())
    op = R.operator_from_problem(ctx, Q, "stencil")
    lmin, lmax, _ = R.lanczos_bounds(ctx, op, None, seed=3, tol=1e-8, which="both")
    ev = np.linalg.eigvalsh(A.toarray())
    assert lmin == pytest.approx(ev[0], rel=1e-5, abs=1e-6)
    assert lmax == pytest.approx(ev[-1], rel=1e-5)
