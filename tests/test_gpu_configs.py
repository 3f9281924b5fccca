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
from rayleighchebyshevgpgpu_b200.verify import stencil_residuals

pytestmark = pytest.mark.gpu


def _solve(ctx, op, P, precision, v0, evecs):
    incr, buf = problems.block_sizes(P.k)
    p = R.make_params(P.k, P.tol, incr=incr, buffer=buf, precision=precision, stop="RESIDUAL_ONLY")
    p.v0_cols = incr + buf
    return R.solve(ctx, op, p, v0=v0, host=False, evecs_out=evecs)


def _check(ctx, op, P, res, evecs, tol):
    k = P.k
    assert res.info["found"] == k
    assert np.all(np.diff(res.evals) >= -1e-12 * np.abs(res.evals[1:]))
    X = evecs[:k]  # rows are eigenvectors (column-major n x k block)
    rel = stencil_residuals(P, X, res.evals)
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
    # both configurations refine with the correction filter (configuration 3: complex blocks)
    assert mixed.info["correction_iterations"] > 0 and mixed.info["fp64_degree_steps"] == 0
    del v0, evecs
    op.close()
    torch.cuda.empty_cache()
