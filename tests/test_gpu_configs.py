"""Whole solves at the full sizes of the benchmark configurations, checked through properties that
do not need a dense oracle: every returned pair satisfies the requested residual (recomputed here
with the stencil written out in plain torch arithmetic on the grid, independent of the library's
kernels), the eigenvectors are orthonormal, the eigenvalues are ascending, and the mixed-precision
solve agrees with the FP64 solve of the same operator and start block to 1e-10 relative."""
import numpy as np
import pytest
import torch

from rayleighchebyshevgpgpu_b200 import problems
from rayleighchebyshevgpgpu_b200 import runtime as R

pytestmark = pytest.mark.gpu


def _solve(ctx, op, P, precision, v0, evecs):
    incr, buf = problems.block_sizes(P.k)
    p = R.make_params(P.k, P.tol, incr=incr, buffer=buf, precision=precision, stop="RESIDUAL_ONLY")
    p.v0_cols = incr + buf
    return R.solve(ctx, op, p, v0=v0, host=False, evecs_out=evecs)


def stencil_apply(P, X):
    """A X for the rows of X (k x n), the Dirichlet stencil of P in torch arithmetic: diag * x plus
    offdiag times every neighbour on the grid (zero padding at the boundary); for complex P the
    y-bonds carry exp(+i 2 pi flux x) from (x, y-1) and its conjugate from (x, y+1)."""
    k = X.shape[0]
    nx, ny, nz = P.nx, P.ny, P.nz
    Xg = X.reshape(k, nz, ny, nx)
    Xp = torch.nn.functional.pad(Xg, (1, 1, 1, 1, 1, 1)) if not X.is_complex() else torch.complex(
        torch.nn.functional.pad(Xg.real, (1, 1, 1, 1, 1, 1)), torch.nn.functional.pad(Xg.imag, (1, 1, 1, 1, 1, 1)))
    diag = torch.from_numpy(P.diag).to(X.device).reshape(nz, ny, nx)
    out = Xg * diag
    if P.kind == 27:
        offs = [(dz, dy, dx) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1) if (dz, dy, dx) != (0, 0, 0)]
    else:
        offs = [(-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1)]
    for dz, dy, dx in offs:
        nb = Xp[:, 1 + dz:1 + dz + nz, 1 + dy:1 + dy + ny, 1 + dx:1 + dx + nx]
        if X.is_complex() and dy != 0 and dx == 0 and dz == 0:
            th = 2.0 * np.pi * P.flux * torch.arange(nx, device=X.device, dtype=torch.float64)
            ph = torch.polar(torch.ones_like(th), th if dy < 0 else -th)
            nb = nb * ph
        out = out + P.offdiag * nb
    return out.reshape(k, -1)


def _check(ctx, op, P, res, evecs, tol):
    k = P.k
    assert res.info["found"] == k
    assert np.all(np.diff(res.evals) >= -1e-12 * np.abs(res.evals[1:]))
    X = evecs[:k]  # rows are eigenvectors (column-major n x k block)
    rel = np.empty(k)
    for c0 in range(0, k, 8):  # a few columns at a time: the padded grid copies stay small
        Xc = X[c0:c0 + 8]
        lam = torch.from_numpy(res.evals[c0:c0 + 8]).to(X.device)
        if X.is_complex():
            lam = lam.to(X.dtype)
        r = torch.linalg.vector_norm(stencil_apply(P, Xc) - lam[:, None] * Xc, dim=1).cpu().numpy()
        rel[c0:c0 + 8] = r / np.maximum(np.abs(res.evals[c0:c0 + 8]), 0.1)
    assert rel.max() <= 1.5 * tol, rel.max()
    G = X.conj() @ X.T
    eye = torch.eye(k, dtype=G.dtype, device=G.device)
    assert torch.linalg.matrix_norm(G - eye, ord=2).item() < 1e-12


@pytest.mark.parametrize("config", [5, 3])
def test_full_size_config_properties(ctx, config):
    P = problems.config5() if config == 5 else problems.config3()
    incr, buf = problems.block_sizes(P.k)
    op = R.operator_from_problem(ctx, P, "stencil")
    v0 = torch.from_numpy(P.start_block(incr + buf)).cuda()
    evecs = torch.empty((P.k, P.n), dtype=v0.dtype, device="cuda")
    mixed = _solve(ctx, op, P, "mixed", v0, evecs)
    _check(ctx, op, P, mixed, evecs, P.tol)
    fp64 = _solve(ctx, op, P, "fp64", v0, evecs)
    _check(ctx, op, P, fp64, evecs, P.tol)
    np.testing.assert_allclose(mixed.evals, fp64.evals, rtol=1e-10)
    if config == 5:
        assert mixed.info["correction_iterations"] > 0 and mixed.info["fp64_degree_steps"] == 0
    del v0, evecs
    op.close()
    torch.cuda.empty_cache()
