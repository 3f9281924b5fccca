"""The reference's own FP64 GPU solver (RayleighChebyshevLMCuda with cuSOLVER QR, cuBLAS products, host
LAPACK eigensolve and a cuSPARSE operator; oracle/ref_gpu_solve.cu, built from the reference's sources)
against this library on the same operator, start block, block sizes and stop test. Both must find the
same eigenvalues to 1e-10 relative and agree with dense LAPACK. Skipped where the driver was not built
(it needs the reference sources at build time)."""
import os
import tempfile

import numpy as np
import pytest

from oracle import rc_oracle as O
from oracle import ref_io
from rayleighchebyshevgpgpu_b200 import problems
from rayleighchebyshevgpgpu_b200 import runtime as R

pytestmark = pytest.mark.gpu


@pytest.mark.skipif(not os.path.exists(ref_io.GPU_SOLVE_BIN), reason="oracle/_ref/ref_gpu_solve not built")
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_reference_gpu_solver_agrees_with_library(ctx, precision):
    P = problems.config1()
    incr, buf = problems.block_sizes(P.k)
    s = incr + buf
    start = P.start_block(s)
    rp, ci, v = P.csr()
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "c1.bin")
        ref_io.write_problem(path, rp, ci, v, start=start)
        ref = ref_io.run_gpu_solve(path, P.k, incr, buf, P.tol, repeats=1, timeout=600)
    assert ref["found"] >= P.k
    ev_ref = np.asarray(ref["evals"][:P.k])
    op = R.operator_from_problem(ctx, P, "csr")
    p = R.make_params(P.k, P.tol, incr=incr, buffer=buf, precision=precision, stop="RESIDUAL_ONLY")
    res = R.solve(ctx, op, p, v0=start, host=True)
    np.testing.assert_allclose(res.evals, ev_ref, rtol=1e-10)
    np.testing.assert_allclose(ev_ref, O.dense_lowest(O.csr_matrix(rp, ci, v), P.k), rtol=1e-10)
    op.close()
