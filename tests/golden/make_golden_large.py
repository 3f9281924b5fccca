"""Generate the large-problem golden fixtures by running the reference's own CPU solver.

The reference's RayleighChebyshevLM::getMinEigenSystem (RayleighChebyshevLM.h:712), compiled from
its sources into oracle/_ref by oracle/Makefile, is run once on each problem below with the same
operator, start block, Lanczos start vector, block sizes and stop test as the GPU tests and the
benchmark use. The reference CPU solve at 128^3 takes on the order of an hour on 8 host threads,
so these fixtures are generated once and committed:

  config2_solve.json  3D 7-point Dirichlet Laplacian 128^3 + U[0,4) potential (seed 2), k = 64,
                      incr 64 + buffer 32, start block N(0,1) seed 3, Lanczos start U[-1,1) seed 11,
                      tol 1e-10, RESIDUAL_ONLY  (the benchmark workload)
  mid3d_solve.json    the same operator family on 64^3 (potential seed 2), k = 32, incr 32 +
                      buffer 16, start block N(0,1) seed 3, Lanczos start U[-1,1) seed 11,
                      tol 1e-10, RESIDUAL_ONLY

Run from the repository root:  python tests/golden/make_golden_large.py [mid3d] [config2]
"""
from __future__ import annotations

import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref_io  # noqa: E402
from rayleighchebyshevgpgpu_b200 import problems  # noqa: E402

CASES = {
    # name: (grid side, eigenpair count)
    "mid3d": (64, 32),
    "config2": (128, 64),
}


def run_case(name: str, threads: int) -> dict:
    side, k = CASES[name]
    P = problems.config2(side)
    P.k = k
    rp, ci, v = P.csr()
    incr, buf = problems.block_sizes(k)
    s = incr + buf
    start = P.start_block(s)
    lz0 = np.random.default_rng(11).uniform(-1.0, 1.0, P.n)
    tmp = tempfile.mkdtemp()
    path = os.path.join(tmp, f"{name}.bin")
    ref_io.write_problem(path, rp, ci, v, start, lz0)
    del start
    r = ref_io.run_ref("solve", path, timeout=6 * 3600, k=k, tol=1e-10, incr=incr, buffer=buf,
                       stop="RESIDUAL_ONLY", threads=threads)
    os.remove(path)
    out = {"problem": f"3D 7-point Dirichlet Laplacian {side}^3 + U[0,4) potential (seed 2)",
           "side": side, "n": P.n, "nnz": int(ci.size), "k": k, "tol": 1e-10, "incr": incr, "buffer": buf,
           "stop": "RESIDUAL_ONLY", "start_block": "N(0,1) seed 3", "lanczos_start": "U[-1,1) seed 11",
           "eigenvalues": r["eigenvalues"], "residuals": r["residuals"], "found": r["found"],
           "count_opapply": r["count_opapply"], "count_ortho": r["count_ortho"],
           "count_eigenvalue": r["count_eigenvalue"], "min_eig_est": r["min_eig_est"],
           "max_eig_est": r["max_eig_est"], "reference_seconds": r["seconds"], "reference_threads": r["threads"]}
    json.dump(out, open(os.path.join(HERE, f"{name}_solve.json"), "w"), indent=1)
    return out


def main():
    ref_io.build_ref()
    names = [a for a in sys.argv[1:] if a in CASES] or list(CASES)
    threads = os.cpu_count() or 1
    for name in names:
        r = run_case(name, threads)
        print(name, "found", r["found"], "in", r["reference_seconds"], "s on", r["reference_threads"], "threads",
              flush=True)


if __name__ == "__main__":
    main()
