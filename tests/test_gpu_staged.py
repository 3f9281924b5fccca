"""The staged degree step (rc_staged.cuh: operands copied to shared memory by asynchronous 16-byte
copies several chunks ahead, persistent CTAs) against the per-row gather kernel it replaces
(rm_step_rows), on the GPU through the C ABI. Both compute every row with the same products
in the same order, so their outputs must be equal bit for bit: single steps (rc_filter_step_rm) on
CSR, 5- and 7-point stencils, real and complex, FP64 and FP32 storage, with and without x_{k-2}, block
widths 5, 24 and 96 and row counts that leave a partial last chunk; whole filter applications
(rc_filter); the bfloat16 correction filter (rc_filter_correction). The context knob RCB200_STAGED=0
selects the per-row kernels. The staged kernel must actually run (its launch counter moves), and an
operator with many distinct column offsets must fall back to the per-row kernel."""
import os

import numpy as np
import pytest

from oracle import rc_oracle as O
from rayleighchebyshevgpgpu_b200 import problems
from rayleighchebyshevgpgpu_b200 import runtime as R

pytestmark = pytest.mark.gpu


def _ctx(staged: bool):
    old = os.environ.get("RCB200_STAGED")
    os.environ["RCB200_STAGED"] = "1" if staged else "0"
    try:
        return R.Context(0)
    finally:
        if old is None:
            os.environ.pop("RCB200_STAGED", None)
        else:
            os.environ["RCB200_STAGED"] = old


@pytest.fixture(scope="module")
def pair():
    a, b = _ctx(True), _ctx(False)
    yield a, b
    a.close()
    b.close()


def _problems():
    rng = np.random.default_rng(3)
    d7 = (20, 17, 13)
    p7 = problems.Problem("s7", d7, 7, 6.0 + rng.uniform(0, 3, int(np.prod(d7))), -1.0)
    d5 = (67, 45)
    p5 = problems.Problem("s5", d5, 5, 4.0 + rng.uniform(0, 3, int(np.prod(d5))), -1.0)
    pc = problems.small_laplacian((12, 11, 10), seed=4, complex_=True, flux=0.11)
    return {"s7": p7, "s5": p5, "c7": pc}


PROBS = _problems()


def _block(n, ld, s, prec, complex_, seed):
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    if complex_:
        dt = torch.complex128 if prec == "fp64" else torch.complex64
        X = torch.randn((n, ld), dtype=dt, device="cuda", generator=g)
    else:
        dt = torch.float64 if prec == "fp64" else torch.float32
        X = torch.randn((n, ld), dtype=dt, device="cuda", generator=g)
    return X


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("s", [5, 24, 96])
@pytest.mark.parametrize("name,form", [("s7", "csr"), ("s7", "stencil"), ("s5", "csr"), ("s5", "stencil"),
                                       ("c7", "csr"), ("c7", "stencil")])
def test_staged_step_equals_per_row_kernel_bitwise(pair, name, form, s, prec):
    import torch
    cs, cu = pair
    P = PROBS[name]
    ops = R.operator_from_problem(cs, P, form), R.operator_from_problem(cu, P, form)
    ld = R.rm_leading_dim(P.complex_, prec, s)
    x = _block(P.n, ld, s, prec, P.complex_, 1)
    z = _block(P.n, ld, s, prec, P.complex_, 2)
    alpha, beta, gamma = (-0.31 + 0.05j, 1.7, -1.0) if P.complex_ else (-0.31, 1.7, -1.0)
    for use_z in (True, False):
        ys = z.clone() if use_z else torch.zeros_like(x)
        yu = z.clone() if use_z else torch.zeros_like(x)
        torch.cuda.synchronize()  # the library works on its own stream
        before = cs.counter("staged_launches")
        R.filter_step_rm(cs, ops[0], x, ys if use_z else None, ys, s, alpha, beta, gamma, prec, ld=ld)
        R.filter_step_rm(cu, ops[1], x, yu if use_z else None, yu, s, alpha, beta, gamma, prec, ld=ld)
        cs.synchronize()
        cu.synchronize()
        assert cs.counter("staged_launches") == before + 1
        assert cu.counter("staged_launches") == 0
        assert torch.equal(ys, yu), (ys - yu).abs().max().item()
    for op in ops:
        op.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("form", ["csr", "stencil"])
def test_staged_filter_equals_per_row_kernel_bitwise(pair, form, prec):
    import torch
    cs, cu = pair
    P = PROBS["s7"]
    ops = R.operator_from_problem(cs, P, form), R.operator_from_problem(cu, P, form)
    X0 = torch.randn((48, P.n), dtype=torch.float64, device="cuda")
    Xs, Xu = X0.clone(), X0.clone()
    torch.cuda.synchronize()  # the library works on its own stream
    R.filter_block(cs, ops[0], Xs, 48, 17, -0.21, 1.8, precision=prec)
    R.filter_block(cu, ops[1], Xu, 48, 17, -0.21, 1.8, precision=prec)
    cs.synchronize()
    cu.synchronize()
    assert torch.equal(Xs, Xu)
    A = O.csr_matrix(*P.csr())
    ref = O.filter_block(A, X0.cpu().numpy().T, 17, -0.21, 1.8)
    tol = 1e-12 if prec == "fp64" else 1e-5
    assert np.abs(Xs.cpu().numpy().T - ref).max() <= tol * np.abs(ref).max()
    for op in ops:
        op.close()


def test_staged_correction_filter_equals_per_row_kernel_bitwise(pair):
    import torch
    cs, cu = pair
    P = PROBS["s7"]
    A = O.csr_matrix(*P.csr())
    w, U = np.linalg.eigh(A.toarray())
    s, m = 40, 11
    rng = np.random.default_rng(7)
    V, _ = np.linalg.qr(U[:, :s] + 1e-5 * rng.standard_normal((P.n, s)))
    H = V.T @ (A @ V)
    lam, Q = np.linalg.eigh(0.5 * (H + H.T))
    Y = V @ Q
    a = -4.0 / (w[-1] - w[s])
    b = 2.0 - a * w[s]
    for form in ("csr", "stencil"):
        ops = R.operator_from_problem(cs, P, form), R.operator_from_problem(cu, P, form)
        Vs = torch.from_numpy(np.ascontiguousarray(Y.T)).cuda()
        Vu = Vs.clone()
        torch.cuda.synchronize()  # the library works on its own stream
        before = cs.counter("staged_launches")
        R.filter_correction(cs, ops[0], Vs, s, lam, m, a / b, b)
        R.filter_correction(cu, ops[1], Vu, s, lam, m, a / b, b)
        assert cs.counter("staged_launches") == before + (m - 1)
        assert torch.equal(Vs, Vu)
        for op in ops:
            op.close()


def test_many_offsets_fall_back_to_the_per_row_kernel(pair):
    import scipy.sparse as sp
    import torch
    cs, cu = pair
    n = 3000
    M = sp.random(n, n, density=0.004, random_state=5, format="csr")
    M = (M + M.T + sp.identity(n) * 3.0).tocsr()
    M.sort_indices()
    ops = [R.CsrOperator(c, M.indptr, M.indices, M.data) for c in (cs, cu)]
    ld = R.rm_leading_dim(False, "fp64", 24)
    x = torch.randn((n, ld), dtype=torch.float64, device="cuda")
    ys, yu = torch.zeros_like(x), torch.zeros_like(x)
    torch.cuda.synchronize()  # the library works on its own stream
    before = cs.counter("staged_launches")
    R.filter_step_rm(cs, ops[0], x, None, ys, 24, 1.0, 0.0, 0.0, "fp64", ld=ld)
    R.filter_step_rm(cu, ops[1], x, None, yu, 24, 1.0, 0.0, 0.0, "fp64", ld=ld)
    cs.synchronize()
    cu.synchronize()
    assert cs.counter("staged_launches") == before
    assert torch.equal(ys, yu)
    ref = M @ x[:, :24].cpu().numpy()
    assert np.abs(ys[:, :24].cpu().numpy() - ref).max() < 1e-12 * np.abs(ref).max()
    for op in ops:
        op.close()
