"""Run one solve of a benchmark configuration and print its result summary as JSON.

  python -m rayleighchebyshevgpgpu_b200.solve_case --config 2 --side 64 --precision mixed --form csr

Useful on its own and as a small, bounded target for profilers (one solve per --repeat).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import problems
from . import runtime as R


def make_problem(config: int, side: int | None, k: int | None):
    if config == 1:
        P = problems.config1()
    elif config == 2:
        P = problems.config2(side or 128)
    elif config == 3:
        P = problems.config3(side or 96, k or 128)
    elif config == 5:
        P = problems.config5(side or 256)
    else:
        raise SystemExit("config must be 1, 2, 3 or 5")
    if k:
        P.k = k
    return P


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", type=int, default=2)
    ap.add_argument("--side", type=int, default=None)
    ap.add_argument("--k", type=int, default=None)
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--form", default="csr", choices=["csr", "stencil"])
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--filter-only", type=int, default=0,
                    help="apply the filter of this degree to the start block instead of solving")
    a = ap.parse_args(argv)
    P = make_problem(a.config, a.side, a.k)
    incr, buf = problems.block_sizes(P.k)
    ctx = R.Context(0)
    op = R.operator_from_problem(ctx, P, a.form)
    v0 = P.start_block(incr + buf)
    if a.filter_only:
        import torch
        X = torch.from_numpy(v0).cuda()
        g1, g2 = R.cpoly_gammas(a.filter_only, 16.0, -0.5)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        stream = torch.cuda.Stream()
        torch.cuda.set_stream(stream)
        ctx.set_stream(stream.cuda_stream)
        times = []
        for _ in range(a.repeat):
            ev0.record()
            R.filter_block(ctx, op, X, incr + buf, a.filter_only, g1, g2, a.precision)
            ev1.record()
            torch.cuda.synchronize()
            times.append(ev0.elapsed_time(ev1) / a.filter_only)
        print(json.dumps({"problem": P.name, "n": P.n, "s": incr + buf, "degree": a.filter_only,
                          "precision": a.precision, "form": a.form, "ms_per_step": times}))
        op.close()
        ctx.close()
        return
    out = []
    for _ in range(a.repeat):
        p = R.make_params(P.k, P.tol, incr=incr, buffer=buf, precision=a.precision, stop="RESIDUAL_ONLY",
                          phase_timing=1, verbose=1 if a.verbose else 0)
        t0 = time.perf_counter()
        res = R.solve(ctx, op, p, v0=v0, host=True, want_vectors=False)
        dt = time.perf_counter() - t0
        out.append({"wall_s": dt, "found": res.info["found"], "eig_min": float(res.evals.min()),
                    "eig_max": float(res.evals.max()),
                    "max_rel_residual": float(np.max(res.residuals / np.maximum(np.abs(res.evals), 0.1))),
                    "info": res.info})
    print(json.dumps({"problem": P.name, "n": P.n, "k": P.k, "precision": a.precision, "form": a.form,
                      "runs": out}))
    op.close()
    ctx.close()


if __name__ == "__main__":
    main()
