"""Time the reference's own FP64 GPU solver (oracle/_ref/ref_gpu_solve: RayleighChebyshevLMCuda with
cuSOLVER QR, cuBLAS products, host LAPACK eigensolve and a cuSPARSE CSR operator) beside this library's
FP64 and mixed solves on the same operator, start block, block sizes and RESIDUAL_ONLY stop test.
A baseline run by hand on a GPU box (test infrastructure; the library never runs it):

    python -m oracle.ref_gpu_baseline --config 2 [--repeats 1]

Prints one JSON line: the reference's wall time per solve (device synchronised around its
getMinEigenSystem) and its own TIMING_ buckets and counts; this library's times on CUDA events for the
same problem; the largest relative eigenvalue difference between the two.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import tempfile

import numpy as np


def main(argv=None):
    import torch

    from oracle import ref_io
    from rayleighchebyshevgpgpu_b200 import problems
    from rayleighchebyshevgpgpu_b200 import runtime as R

    ap = argparse.ArgumentParser()
    ap.add_argument("--config", type=int, default=2, choices=[1, 2])
    ap.add_argument("--repeats", type=int, default=1)
    a = ap.parse_args(argv)
    P = problems.config1() if a.config == 1 else problems.config2()
    incr, buf = problems.block_sizes(P.k)
    s = incr + buf
    start = P.start_block(s)
    rp, ci, v = P.csr()
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "problem.bin")
        ref_io.write_problem(path, rp, ci, v, start=start)
        ref = ref_io.run_gpu_solve(path, P.k, incr, buf, P.tol, repeats=a.repeats, timeout=3600)
    ctx = R.Context(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    op = R.CsrOperator(ctx, rp, ci, v)
    v0 = torch.from_numpy(start).cuda()
    evecs = torch.empty((P.k, P.n), dtype=torch.float64, device="cuda")
    ours = {}
    for prec in ("fp64", "mixed"):
        times = []
        res = None
        for i in range(a.repeats + 1):  # the first solve is a warm-up
            p = R.make_params(P.k, P.tol, incr=incr, buffer=buf, precision=prec, stop="RESIDUAL_ONLY")
            p.v0_cols = s
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            res = R.solve(ctx, op, p, v0=v0, host=False, evecs_out=evecs)
            e1.record(stream)
            torch.cuda.synchronize()
            if i > 0:
                times.append(e0.elapsed_time(e1) * 1e-3)
        ours[prec] = {"wall_s": times, "inner_iterations": res.info["inner_iterations"],
                      "degree_steps": res.info["degree_steps"],
                      "max_rel_eig_diff_vs_reference_gpu": float(
                          np.max(np.abs(res.evals - np.asarray(ref["evals"][:P.k])) / np.abs(res.evals)))}
    out = {"config": a.config, "n": P.n, "k": P.k, "subspace": s, "tol": P.tol,
           "reference_gpu": {"wall_s": ref["wall_s"], "found": ref["found"], "timing": ref["timing"],
                             "counts": ref["counts"]},
           "ours": ours,
           "speedup_vs_reference_gpu": {prec: statistics.median(ref["wall_s"]) / statistics.median(ours[prec]["wall_s"])
                                        for prec in ours}}
    print(json.dumps(out), flush=True)
    op.close()
    ctx.close()


if __name__ == "__main__":
    main()
