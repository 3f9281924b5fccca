"""Serving workload (configuration 4) through the request server.

256 requests of random-potential Laplacians (2D 5-point or 3D 7-point stencils, n log-uniform in
[1e4, 2e6], k in {8, 16, 32, 64}, tol in {1e-8, 1e-10}; problems.serve_stream) with the FP32
filter and FP64 Rayleigh-Ritz (RC_PREC_MIXED), RESIDUAL_ONLY stop test.

Two passes over the same requests:
  capacity  every request submitted at t = 0; capacity = requests / wall time (saturated server)
  poisson   request i submitted at its Poisson arrival time, mean rate = rate_frac * capacity;
            latency = submit -> finished (rc_request_info), p50 / p99 over the requests
Throughput is eigenpairs per second of wall time (sum of k over the requests / makespan).

  python -m rayleighchebyshevgpgpu_b200.serve_bench [--count 256] [--max-active 16] [--rate-frac 0.8]
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import problems
from . import runtime as R


def _params(P, i):
    p = R.make_params(P.k, P.tol, precision="mixed", stop="RESIDUAL_ONLY")
    p.seed = 1000 + i
    return p


def _pass(srv, stream, ops, arrivals=None):
    """Submit the stream (at `arrivals` seconds from the start, or all at once); wait for all."""
    t0 = time.perf_counter()
    handles = []
    for i, (rq, op) in enumerate(zip(stream, ops)):
        if arrivals is not None:
            delay = arrivals[i] - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
        handles.append(srv.submit(op, _params(rq.problem, i), want_vectors=False))
    states = [h.wait(600000.0) for h in handles]
    wall = time.perf_counter() - t0
    infos = [h.info() for h in handles]
    found = []
    for h, st in zip(handles, states):
        found.append(h.result().info["found"] if st == "done" else 0)
        h.release()
    lat = np.array([q["latency_ms"] for q in infos])
    return {
        "wall_s": wall,
        "done": int(sum(st == "done" for st in states)),
        "eigenpairs": int(sum(found)),
        "latency_ms": lat,
        "queue_ms": np.array([q["queue_ms"] for q in infos]),
        "batches": np.array([q["batches"] for q in infos]),
    }


def run(count: int = 256, max_active: int = 16, rate_frac: float = 0.8, use_graphs: bool = True,
        device: int = 0, warmup: int = 4) -> dict:
    stream = problems.serve_stream(count)
    ctx = R.Context(device)
    ops = [R.StencilOperator(ctx, rq.problem.kind, rq.problem.dims, rq.problem.diag, rq.problem.offdiag)
           for rq in stream]
    srv = R.Server(device, max_active=max_active, use_graphs=use_graphs)
    try:
        # warm-up on the smallest requests (first graph builds, pool growth)
        small = sorted(range(count), key=lambda i: stream[i].problem.n)[:warmup]
        _pass(srv, [stream[i] for i in small], [ops[i] for i in small])
        cap = _pass(srv, stream, ops)
        capacity = cap["done"] / cap["wall_s"]
        rate = rate_frac * capacity
        arrivals = np.cumsum([rq.arrival_gap for rq in stream]) / rate
        arrivals -= arrivals[0]
        st0 = srv.stats()
        poi = _pass(srv, stream, ops, arrivals)
        st1 = srv.stats()
    finally:
        srv.close()
        for op in ops:
            op.close()
        ctx.close()
    lat = poi["latency_ms"]
    total_k = sum(rq.problem.k for rq in stream)
    return {
        "requests": count,
        "completed": poi["done"],
        "eigenpairs": poi["eigenpairs"],
        "eigenpairs_per_s": poi["eigenpairs"] / poi["wall_s"],
        "requests_per_s": poi["done"] / poi["wall_s"],
        "latency_ms_p50": float(np.percentile(lat, 50)),
        "latency_ms_p99": float(np.percentile(lat, 99)),
        "latency_ms_mean": float(lat.mean()),
        "queue_ms_p50": float(np.percentile(poi["queue_ms"], 50)),
        "queue_ms_p99": float(np.percentile(poi["queue_ms"], 99)),
        "makespan_s": poi["wall_s"],
        "capacity_requests_per_s": capacity,
        "capacity_eigenpairs_per_s": cap["eigenpairs"] / cap["wall_s"],
        "arrival_rate_per_s": rate,
        "sum_k": total_k,
        "max_active": max_active,
        "batches": st1["batches"] - st0["batches"],
        "batched_filter_applications": st1["batched_jobs"] - st0["batched_jobs"],
        "max_jobs_in_batch": st1["max_jobs_in_batch"],
        "graph_launches": st1["graph_launches"] - st0["graph_launches"],
        "graphs_built": st1["graphs_built"],
        "hbm_budget_bytes": st1["budget"],
        "hbm_peak_reserved_bytes": st1["bytes_peak"],
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--count", type=int, default=256)
    ap.add_argument("--max-active", type=int, default=16)
    ap.add_argument("--rate-frac", type=float, default=0.8)
    ap.add_argument("--no-graphs", action="store_true")
    a = ap.parse_args()
    print(json.dumps(run(a.count, a.max_active, a.rate_frac, not a.no_graphs)), flush=True)


if __name__ == "__main__":
    main()
