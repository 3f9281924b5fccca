"""Generate the golden fixtures of tests/golden/ by running the reference's own CPU code.

The reference ships no tests or golden vectors, so the fixtures come from the reference
compiled from its sources (oracle/_ref, built by oracle/Makefile from the reference headers):

  cpoly.json          XStar / UpperXStar for m = 1..200 and two getStarDegreeAndSpectralRadius
                      queries (LanczosCpoly.h)
  config1_solve.json  RayleighChebyshevLM::getMinEigenSystem on configuration 1 (2D 5-point
                      Laplacian 64x64 + U[0,1) potential, k=16, tol=1e-10, RESIDUAL_ONLY), with the
                      start block N(0,1) seed 1 and Lanczos start vector U[-1,1) seed 11, plus the
                      dense LAPACK eigenvalues
  filter_small.npz    LanczosCpolyOperatorLM::apply on a 16x16 Laplacian (+U[0,1) potential,
                      seed 21), 3 columns N(0,1) seed 22, degree 12
  lanczos_config1.json  LanczosMaxMinFinder::getMinMaxEigenvalues (max stop) on configuration 1

Run from the repository root:  python tests/golden/make_golden.py
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

from oracle import rc_oracle as O  # noqa: E402
from oracle import ref_io  # noqa: E402
from rayleighchebyshevgpgpu_b200 import problems  # noqa: E402


def main():
    ref_io.build_ref()
    tmp = tempfile.mkdtemp()
    # --- polynomial design
    cp = ref_io.run_ref("cpoly", None, mmax=200, shift=-0.5, bound=8.0, star=0.9, degmax=200)
    cp2 = ref_io.run_ref("cpoly", None, mmax=1, shift=-0.42, bound=8.55, star=0.43, degmax=200)
    cp3 = ref_io.run_ref("cpoly", None, mmax=1, shift=-1.0, bound=17.0, star=6.0, degmax=200)
    json.dump({"xstar": cp["xstar"], "upper_xstar": cp["upper_xstar"],
               "queries": [
                   {"shift": -0.5, "bound": 8.0, "star": 0.9, "degmax": 200,
                    "star_degree": cp["star_degree"], "star_bound": cp["star_bound"]},
                   {"shift": -0.42, "bound": 8.55, "star": 0.43, "degmax": 200,
                    "star_degree": cp2["star_degree"], "star_bound": cp2["star_bound"]},
                   {"shift": -1.0, "bound": 17.0, "star": 6.0, "degmax": 200,
                    "star_degree": cp3["star_degree"], "star_bound": cp3["star_bound"]}]},
              open(os.path.join(HERE, "cpoly.json"), "w"), indent=1)

    # --- configuration 1 whole solve
    P = problems.config1()
    rp, ci, v = P.csr()
    incr, buf = problems.block_sizes(P.k)
    s = incr + buf
    start = P.start_block(s)
    lz0 = np.random.default_rng(11).uniform(-1.0, 1.0, P.n)
    path = os.path.join(tmp, "c1.bin")
    ref_io.write_problem(path, rp, ci, v, start, lz0)
    r = ref_io.run_ref("solve", path, k=P.k, tol=1e-10, incr=incr, buffer=buf, stop="RESIDUAL_ONLY")
    dense = O.dense_lowest(O.csr_matrix(rp, ci, v), P.k)
    json.dump({"k": P.k, "tol": 1e-10, "incr": incr, "buffer": buf, "stop": "RESIDUAL_ONLY",
               "eigenvalues": r["eigenvalues"], "residuals": r["residuals"], "found": r["found"],
               "count_opapply": r["count_opapply"], "dense_eigenvalues": dense.tolist(),
               "min_eig_est": r["min_eig_est"], "max_eig_est": r["max_eig_est"]},
              open(os.path.join(HERE, "config1_solve.json"), "w"), indent=1)
    lz = ref_io.run_ref("lanczos", path, tol=1e-6, which="max")
    json.dump(lz, open(os.path.join(HERE, "lanczos_config1.json"), "w"), indent=1)

    # --- small filter application
    Q = problems.small_laplacian((16, 16), seed=21)
    rp, ci, v = Q.csr()
    X = np.random.default_rng(22).standard_normal((3, Q.n))
    path = os.path.join(tmp, "f.bin")
    ref_io.write_problem(path, rp, ci, v, X)
    out = os.path.join(tmp, "f.out")
    degree, bound, shift = 12, 9.0, -0.3
    ref_io.run_ref("filter", path, degree=degree, bound=bound, shift=shift, reps=1, out=out)
    Y = np.fromfile(out, dtype=np.float64).reshape(3, Q.n)
    np.savez_compressed(os.path.join(HERE, "filter_small.npz"), X=X, Y=Y, degree=degree, bound=bound, shift=shift)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
