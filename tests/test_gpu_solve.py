"""Whole-solve parity on the GPU through rc_solve: eigenvalues against the reference's own
CPU solver (golden) and dense LAPACK, residuals against the requested tolerance."""
import ctypes as C
import json
import os

import numpy as np
import pytest

from oracle import rc_oracle as O
from rayleighchebyshevgpgpu_b200 import _capi
from rayleighchebyshevgpgpu_b200 import problems
from rayleighchebyshevgpgpu_b200 import runtime as R

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _solve(ctx, op, P, k, tol, precision="fp64", start=None, incr=None, buffer=None, **kw):
    p = R.make_params(k, tol, incr=incr, buffer=buffer, precision=precision, stop="RESIDUAL_ONLY", **kw)
    return R.solve(ctx, op, p, v0=start, host=True)


def _check_pairs(A, res, k, tol, rtol=1e-10):
    dense = O.dense_lowest(A, k)
    assert res.info["found"] == k
    np.testing.assert_allclose(res.evals, dense, rtol=rtol, atol=1e-13)
    X = res.evecs.T  # n x k
    r = np.linalg.norm(A @ X - X * res.evals, axis=0) / np.maximum(np.abs(res.evals), 0.1)
    assert r.max() <= 1.5 * tol, r.max()
    return dense


@pytest.mark.parametrize("orth_mode", [0, 1])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("form", ["csr", "stencil"])
def test_config1_matches_reference_golden(ctx, precision, form, orth_mode):
    g = json.load(open(os.path.join(GOLD, "config1_solve.json")))
    P = problems.config1()
    A = O.csr_matrix(*P.csr())
    op = R.operator_from_problem(ctx, P, form)
    s = g["incr"] + g["buffer"]
    lz0 = np.random.default_rng(11).uniform(-1.0, 1.0, P.n)
    keep = np.ascontiguousarray(lz0)
    res = _solve(ctx, op, P, g["k"], g["tol"], precision, start=P.start_block(s), incr=g["incr"],
                 buffer=g["buffer"], lanczos_v0=keep.ctypes.data, orth_mode=orth_mode)
    np.testing.assert_allclose(res.evals, g["eigenvalues"], rtol=1e-10)
    if orth_mode == 1:
        assert res.info["fused_rr"] == 0
    else:
        assert res.info["fused_rr"] > 0
    _check_pairs(A, res, g["k"], g["tol"])
    assert res.info["lanczos_iterations"] > 0 and res.info["degree_steps"] > 0
    if precision == "mixed":
        assert res.info["mixed_iterations"] >= 1 and res.info["fp64_degree_steps"] < res.info["degree_steps"]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_complex_tight_binding_vs_lapack(ctx, precision):
    Q = problems.small_laplacian((10, 10, 10), seed=9, complex_=True, flux=1.0 / 17.0)
    A = O.csr_matrix(*Q.csr())
    for form in ("csr", "stencil"):
        op = R.operator_from_problem(ctx, Q, form)
        res = _solve(ctx, op, Q, 16, 1e-9, precision, start=Q.start_block(24))
        _check_pairs(A, res, 16, 1e-9, rtol=1e-9)


@pytest.mark.parametrize("kind,dims,k", [(5, (80, 72), 32), (7, (18, 17, 16), 16), (27, (16, 15, 14), 16)])
def test_mixed_correction_filter_matches_fp64(ctx, kind, dims, k):
    """MIXED precision past the switch tolerance runs the correction filter (the recurrence on the
    residual block of the Ritz vectors, bfloat16 storage, FP32 arithmetic): it reaches tol 1e-10 with no FP64 degree step and the
    FP64 path's eigenvalues; mixed_refine = 1 keeps the FP64 refinement filter."""
    n = int(np.prod(dims))
    diag = (4.0 if kind == 5 else (6.0 if kind == 7 else 1.0)) + np.random.default_rng(kind).uniform(0, 3, n)
    Q = problems.Problem(f"corr{kind}", dims, kind, diag, -1.0 / 26.0 if kind == 27 else -1.0, k=k)
    A = O.csr_matrix(*Q.csr())
    dense = O.dense_lowest(A, k)
    incr, buf = problems.block_sizes(k)
    start = Q.start_block(incr + buf)
    for form in ("csr", "stencil"):
        op = R.operator_from_problem(ctx, Q, form)
        f64 = _solve(ctx, op, Q, k, 1e-10, "fp64", start=start)
        mix = _solve(ctx, op, Q, k, 1e-10, "mixed", start=start)
        old = _solve(ctx, op, Q, k, 1e-10, "mixed", start=start, mixed_refine=1)
        assert mix.info["correction_iterations"] > 0, mix.info
        assert mix.info["fp64_degree_steps"] == 0, mix.info
        assert mix.info["correction_degree_steps"] > 0
        assert old.info["correction_iterations"] == 0 and old.info["fp64_degree_steps"] > 0
        np.testing.assert_allclose(mix.evals, f64.evals, rtol=1e-10)
        np.testing.assert_allclose(mix.evals, dense, rtol=1e-10, atol=1e-13)
        X = mix.evecs.T
        r = np.linalg.norm(A @ X - X * mix.evals, axis=0) / np.maximum(np.abs(mix.evals), 0.1)
        assert r.max() <= 1.5e-10, r.max()
        op.close()


@pytest.mark.parametrize("case", ["complex7", "complex5", "wide5"])
def test_mixed_correction_filter_complex_and_wide_blocks(ctx, case):
    """The correction filter on complex Hermitian operators (complex bfloat16 blocks, c64 arithmetic)
    and on real blocks wider than 96 columns (k = 96, s = 144): no FP64 degree step, the FP64 path's
    eigenvalues and dense LAPACK's (zheevr / dsyevr)."""
    if case == "complex7":
        Q = problems.small_laplacian((12, 11, 10), seed=21, complex_=True, flux=1.0 / 17.0)
        k, tol = 32, 1e-9
    elif case == "complex5":
        Q = problems.small_laplacian((48, 44), seed=22, complex_=True, flux=0.11)
        k, tol = 24, 1e-9
    else:
        Q = problems.small_laplacian((60, 50), seed=23, vmax=3.0)
        k, tol = 96, 1e-10
    A = O.csr_matrix(*Q.csr())
    dense = O.dense_lowest(A, k)
    incr, buf = problems.block_sizes(k)
    start = Q.start_block(incr + buf)
    for form in ("csr", "stencil"):
        op = R.operator_from_problem(ctx, Q, form)
        f64 = _solve(ctx, op, Q, k, tol, "fp64", start=start, incr=incr, buffer=buf)
        mix = _solve(ctx, op, Q, k, tol, "mixed", start=start, incr=incr, buffer=buf)
        assert mix.info["correction_iterations"] > 0, mix.info
        assert mix.info["fp64_degree_steps"] == 0, mix.info
        np.testing.assert_allclose(mix.evals, f64.evals, rtol=tol)
        np.testing.assert_allclose(mix.evals, dense, rtol=tol, atol=1e-13)
        X = mix.evecs.T
        r = np.linalg.norm(A @ X - X * mix.evals, axis=0) / np.maximum(np.abs(mix.evals), 0.1)
        assert r.max() <= 1.5 * tol, r.max()
        op.close()


@pytest.mark.parametrize("kind,dims,k", [(7, (18, 17, 16), 24), (27, (14, 13, 12), 16), (5, (70, 66), 40)])
def test_row_major_rayleigh_ritz_matches_column_major(kind, dims, k):
    """After a correction filter the Rayleigh-Ritz step runs on row-major blocks (filtered block and
    W = A V row-major, Gram and Ritz-vector DMMA kernels reading rows); RCB200_RM_RR=0 keeps every
    block column-major. The two differ only in the rounding of W = A V: the same iterations, the same
    eigenvalues to 1e-12, both at the requested residual and equal to dense LAPACK."""
    import os
    n = int(np.prod(dims))
    diag = (4.0 if kind == 5 else (6.0 if kind == 7 else 1.0)) + np.random.default_rng(kind + 50).uniform(0, 3, n)
    Q = problems.Problem(f"rmrr{kind}", dims, kind, diag, -1.0 / 26.0 if kind == 27 else -1.0, k=k)
    A = O.csr_matrix(*Q.csr())
    dense = O.dense_lowest(A, k)
    incr, buf = problems.block_sizes(k)
    start = Q.start_block(incr + buf)
    out = {}
    for flag in ("1", "0"):
        old = os.environ.get("RCB200_RM_RR")
        os.environ["RCB200_RM_RR"] = flag
        try:
            c = R.Context(0)
        finally:
            if old is None:
                os.environ.pop("RCB200_RM_RR", None)
            else:
                os.environ["RCB200_RM_RR"] = old
        for form in ("csr", "stencil"):
            op = R.operator_from_problem(c, Q, form)
            res = _solve(c, op, Q, k, 1e-10, "mixed", start=start)
            assert res.info["correction_iterations"] > 0 and res.info["fp64_degree_steps"] == 0
            X = res.evecs.T
            r = np.linalg.norm(A @ X - X * res.evals, axis=0) / np.maximum(np.abs(res.evals), 0.1)
            assert r.max() <= 1.5e-10, r.max()
            np.testing.assert_allclose(res.evals, dense, rtol=1e-10, atol=1e-13)
            out[(flag, form)] = res
            op.close()
        c.close()
    for form in ("csr", "stencil"):
        a, b = out[("1", form)], out[("0", form)]
        np.testing.assert_allclose(a.evals, b.evals, rtol=1e-12)
        assert abs(a.info["inner_iterations"] - b.info["inner_iterations"]) <= 1


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_multipass_deflation_incr_smaller_than_k(ctx, precision):
    Q = problems.small_laplacian((24, 24), seed=5)
    A = O.csr_matrix(*Q.csr())
    op = R.operator_from_problem(ctx, Q, "csr")
    res = _solve(ctx, op, Q, 12, 1e-10, precision, incr=4, buffer=8)
    assert res.info["outer_passes"] >= 3
    _check_pairs(A, res, 12, 1e-10)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_interval_mode_finds_all_below_lambda_max(ctx, precision):
    Q = problems.small_laplacian((20, 20), seed=6)
    A = O.csr_matrix(*Q.csr())
    dense = np.linalg.eigvalsh(A.toarray())
    lam = 0.5 * (dense[9] + dense[10])  # exactly 10 eigenvalues below
    op = R.operator_from_problem(ctx, Q, "csr")
    p = R.make_params(4, 1e-10, incr=4, buffer=8, precision=precision, stop="RESIDUAL_ONLY", mode=2,
                      lambda_max=lam)
    p.eig_count = Q.n
    res = R.solve(ctx, op, p, host=True)
    np.testing.assert_allclose(np.sort(res.evals), dense[:10], rtol=1e-9)


def test_explicit_bounds_mode(ctx):
    P = problems.config1()
    A = O.csr_matrix(*P.csr())
    op = R.operator_from_problem(ctx, P, "csr")
    p = R.make_params(8, 1e-10, incr=8, buffer=8, stop="RESIDUAL_ONLY", mode=1, min_eig_est=0.4,
                      max_eig_bound=8.6)
    res = R.solve(ctx, op, p, v0=P.start_block(16), host=True)
    _check_pairs(A, res, 8, 1e-10)
    assert res.info["lanczos_iterations"] == 0


def test_device_buffers_equal_host_buffers(ctx):
    import torch
    P = problems.config1()
    op = R.operator_from_problem(ctx, P, "csr")
    s = 24
    start = P.start_block(s)
    a = _solve(ctx, op, P, 16, 1e-10, start=start, incr=16, buffer=8)
    p = R.make_params(16, 1e-10, incr=16, buffer=8, stop="RESIDUAL_ONLY")
    p.v0_cols = s
    v0 = torch.from_numpy(start).cuda()
    ev = torch.zeros((16, P.n), dtype=torch.float64, device="cuda")
    b = R.solve(ctx, op, p, v0=v0, host=False, evecs_out=ev)
    np.testing.assert_array_equal(a.evals, b.evals)
    np.testing.assert_array_equal(a.evecs, ev.cpu().numpy())


def test_repeat_solves_bitwise_deterministic(ctx):
    P = problems.config1()
    op = R.operator_from_problem(ctx, P, "stencil")
    a = _solve(ctx, op, P, 16, 1e-10, "mixed", start=P.start_block(24))
    b = _solve(ctx, op, P, 16, 1e-10, "mixed", start=P.start_block(24))
    np.testing.assert_array_equal(a.evals, b.evals)
    np.testing.assert_array_equal(a.residuals, b.residuals)


def test_callback_operator_foreign_apply(ctx):
    """A user operator behind the reference's apply(in, out, alpha, beta) contract (torch SpMM)."""
    import torch
    Q = problems.small_laplacian((18, 17), seed=13)
    rp, ci, v = Q.csr()
    A = O.csr_matrix(rp, ci, v)
    At = torch.sparse_csr_tensor(torch.from_numpy(rp.astype(np.int64)), torch.from_numpy(ci.astype(np.int64)),
                                 torch.from_numpy(v), size=(Q.n, Q.n)).cuda()
    calls = {"n": 0}

    def apply(pin, pout, n, s, ld, alpha, beta, stream):
        calls["n"] += 1
        torch.cuda.synchronize()
        src = _wrap(pin, n, s)
        dst = _wrap(pout, n, s)
        y = torch.sparse.mm(At, src.T).T
        dst.copy_(alpha.real * y + beta.real * dst)
        torch.cuda.synchronize()
        return 0

    op = R.CallbackOperator(ctx, Q.n, apply)
    res = _solve(ctx, op, Q, 8, 1e-10, start=Q.start_block(16), incr=8, buffer=8)
    assert calls["n"] > 10
    _check_pairs(A, res, 8, 1e-10)


def _wrap(ptr, n, s):
    """View a device pointer as an (s, n) float64 CUDA tensor (column-major n x s block)."""
    import torch

    class _CAI:
        def __init__(self):
            self.__cuda_array_interface__ = {"shape": (s, n), "typestr": "<f8", "data": (ptr, False), "version": 3,
                                             "strides": None}
    return torch.as_tensor(_CAI(), device="cuda")


def test_bad_csr_rejected(ctx):
    rp = np.array([0, 1, 2], dtype=np.int32)
    ci = np.array([0, 5], dtype=np.int32)  # out of range
    with pytest.raises(_capi.RCError) as e:
        R.CsrOperator(ctx, rp, ci, np.array([1.0, 1.0]))
    assert e.value.status == 1


def test_nan_operator_reports_error_not_crash(ctx):
    Q = problems.small_laplacian((12, 12), seed=2)
    rp, ci, v = Q.csr()
    v = v.copy()
    v[7] = np.nan
    op = R.CsrOperator(ctx, rp, ci, v)
    with pytest.raises(_capi.RCError):
        _solve(ctx, op, Q, 4, 1e-10, start=Q.start_block(12), incr=4, buffer=8, max_inner_loop=50)
    # the context stays usable
    good = R.operator_from_problem(ctx, Q, "csr")
    res = _solve(ctx, good, Q, 4, 1e-10, start=Q.start_block(12), incr=4, buffer=8)
    assert res.info["found"] == 4


def test_non_hermitian_complex_detected(ctx):
    Q = problems.small_laplacian((6, 6, 6), seed=3, complex_=True, flux=0.1)
    rp, ci, v = Q.csr()
    v = v.copy()
    v[rp[:-1]] += 0.5j  # imaginary diagonal: not Hermitian
    op = R.CsrOperator(ctx, rp, ci, v)
    with pytest.raises(_capi.RCError) as e:
        R.lanczos_bounds(ctx, op, None, seed=1, tol=1e-6, which="max")
    assert e.value.status == 4
