"""Benchmark: time-to-solution and eigenpairs/s at residual <= 1e-10 on one B200, mixed vs FP64.

Workload (configuration 2): lowest 64 eigenpairs of the 3D 7-point Dirichlet Laplacian on 128^3
(n = 2,097,152; CSR with FP64 values and int32 indices, 14,581,760 nnz) plus a U[0,4) potential
(seed 2); start block N(0,1) (seed 3), subspace 64 + 32 buffer; stop test RESIDUAL_ONLY at 1e-10.
A "step" is one whole solve (Lanczos bounds, filtered subspace iteration, closing FP64 sweep)
from the operator and start block resident in HBM to eigenvalues and residuals on the host.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--side 128]

Multi-GPU: the solve does not shard across GPUs in this build; N processes run N independent
replicas (one per GPU) and the value is the aggregate eigenpairs/s (weak scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "time-to-solution & eigenpairs/s at resid<=1e-10, mixed vs FP64 on 1 B200; p50/p99"
# Degree-steps of a whole FP64 solve of configuration 2 on the GPU path: multiplies the reference CPU
# per-degree-step time into its time-to-solution estimate (the CPU solve itself runs for hours).
# Measured by this bench (fp64 leg, info.degree_steps); refreshed when the solver changes.
CONFIG2_FP64_DEGREE_STEPS = 1659


def profile_dram_bytes_per_row():
    """DRAM bytes per grid row of one filter degree-step, from the committed ncu summaries
    (lines "dram-bytes-per-row fp32=<B> fp64=<B>" and "dram-bytes-per-row corr=<B>"), or None."""
    out = {}
    for name in ("rm_step_kernel_csr_96cube_s96.md", "rm_step_src_kernel_csr_96cube_s96.md"):
        try:
            for line in open(os.path.join(ROOT, "profiles", name)):
                if line.startswith("dram-bytes-per-row"):
                    out.update({k: float(v) for k, v in (t.split("=") for t in line.split()[1:])})
        except (OSError, ValueError):
            pass
    return out if "fp32" in out and "fp64" in out else None


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--side", type=int, default=128)
    ap.add_argument("--fp64-steps", type=int, default=2)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--cpu-sample-degree", type=int, default=4)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serve-count", type=int, default=64,
                    help="requests of the configuration-4 serving stream run after the timed solves (0: skip)")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def config_dict(args, k, incr, buf, n, nnz):
    return {"workload": f"config2: 3D 7-point Laplacian {args.side}^3 + U[0,4) potential, CSR fp64/int32, "
                        f"lowest {k} eigenpairs, tol 1e-10 RESIDUAL_ONLY",
            "n": n, "nnz": nnz, "k": k, "subspace": incr + buf, "increment": incr, "buffer": buf,
            "operator_form": "csr", "start_block": "N(0,1) seed 3",
            "l2": "inputs larger than L2 (start block 1.6 GB, operator 183 MB)"}


# ---------------------------------------------------------------------------------------------
# CPU baseline: the reference's own filter (LanczosCpolyOperatorLM::apply) built from its
# sources (oracle/_ref), a few degree-steps on the full configuration-2 block, all host threads.
# ---------------------------------------------------------------------------------------------
def cpu_reference_sample(P, incr, buf, degree, rp, ci, v):
    from oracle import rc_oracle as O
    from oracle import ref_io
    s = incr + buf
    threads = os.cpu_count() or 1
    start = P.start_block(s)
    if ref_io.ref_available():
        d = tempfile.mkdtemp()
        path = os.path.join(d, "c2.bin")
        ref_io.write_problem(path, rp, ci, v, start)
        lmin, lmax = 0.4, 10.4
        r = ref_io.run_ref("filter", path, degree=degree, bound=lmax, shift=-lmin, reps=1, threads=threads)
        os.remove(path)
        return r["seconds"] / degree, threads, "reference"
    # oracle port (numpy/scipy, single thread BLAS-free SpMM)
    A = O.csr_matrix(rp, ci, v)
    g1, g2 = O.gammas(degree, 10.4, -0.4)
    t0 = time.perf_counter()
    O.filter_block(A, start.T, degree, g1, g2)
    return (time.perf_counter() - t0) / degree, 1, "port"


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from rayleighchebyshevgpgpu_b200 import problems
    P = problems.config2(args.side)
    incr, buf = problems.block_sizes(P.k)
    rp, ci, v = P.csr()
    per_step = []
    kind, threads = "reference", os.cpu_count() or 1
    for i in range(args.warmup + args.steps):
        t, threads, kind = cpu_reference_sample(P, incr, buf, args.cpu_sample_degree, rp, ci, v)
        if i >= args.warmup:
            per_step.append(t)
    t_step = statistics.median(per_step)
    tts = t_step * CONFIG2_FP64_DEGREE_STEPS
    value = P.k / tts
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "eigenpairs/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": tts * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_dict(args, P.k, incr, buf, P.n, len(ci)),
        "cpu_baseline": {"value": value, "unit": "eigenpairs/s", "cores": threads, "kind": kind,
                         "sample": f"{args.cpu_sample_degree} degree-steps of the reference CPU filter "
                                   f"(LanczosCpolyOperatorLM::apply) on the full {incr + buf}-column block, "
                                   f"{t_step * 1e3:.1f} ms/step, x {CONFIG2_FP64_DEGREE_STEPS} degree-steps of a "
                                   f"whole FP64 solve; a lower bound (excludes Lanczos, orthogonalisation, "
                                   f"Rayleigh-Ritz)"},
        "e2e": {"value": value, "unit": "eigenpairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------
# Our arm
# ---------------------------------------------------------------------------------------------
def run_ours(args):
    import torch
    import torch.distributed as dist

    from rayleighchebyshevgpgpu_b200 import problems
    from rayleighchebyshevgpgpu_b200 import replicas
    from rayleighchebyshevgpgpu_b200 import runtime as R

    env = replicas.rank_env()
    world, rank, local = env.world, env.rank, env.local
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        return replicas.max_over_ranks(x, world, device="cuda")

    P = problems.config2(args.side)
    incr, buf = problems.block_sizes(P.k)
    s = incr + buf
    rp, ci, v = P.csr()
    ctx = R.Context(local)
    # an explicit (non-default) stream: the library and the CUDA events must see the same stream
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    op = R.CsrOperator(ctx, rp, ci, v)
    start_host = P.start_block(s)
    v0 = torch.from_numpy(start_host).cuda()
    evecs = torch.empty((P.k, P.n), dtype=torch.float64, device="cuda")
    lz0 = np.ascontiguousarray(np.random.default_rng(11).uniform(-1.0, 1.0, P.n))

    def params(prec):
        p = R.make_params(P.k, P.tol, incr=incr, buffer=buf, precision=prec, stop="RESIDUAL_ONLY",
                          phase_timing=1, lanczos_v0=lz0.ctypes.data)
        p.v0_cols = s
        return p

    def one(prec):
        return R.solve(ctx, op, params(prec), v0=v0, host=False, evecs_out=evecs)

    # ---- warm-up (mixed) ----
    for _ in range(args.warmup):
        one("mixed")
    torch.cuda.synchronize()

    # ---- timed mixed solves ----
    clocks = ClockSampler(local)
    ctx.launches(reset=True)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    times, infos = [], []
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    res_mixed = None
    for _ in range(args.steps):
        ev0.record(stream)
        res_mixed = one("mixed")
        ev1.record(stream)
        torch.cuda.synchronize()
        times.append(ev0.elapsed_time(ev1))
        infos.append(res_mixed.info)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    launches = ctx.launches()
    mixed_vecs = evecs.clone()
    t_mixed = max_over_ranks(statistics.median(times))

    # ---- FP64 path (the plain-FP64 baseline of the same solver) ----
    one("fp64")
    torch.cuda.synchronize()
    t64, info64, res64 = [], None, None
    for _ in range(args.fp64_steps):
        ev0.record(stream)
        res64 = one("fp64")
        ev1.record(stream)
        torch.cuda.synchronize()
        t64.append(ev0.elapsed_time(ev1))
        info64 = res64.info
    t_fp64 = max_over_ranks(statistics.median(t64)) if t64 else None
    fp64_vecs = evecs.clone()

    # ---- accuracy: mixed vs FP64 (eigenvalues and largest subspace angle) ----
    eig_err = float(np.max(np.abs(res_mixed.evals - res64.evals) / np.abs(res64.evals))) if res64 else None
    with torch.no_grad():
        # largest principal angle between the two k-dimensional eigenspaces: sin(theta_max) is the
        # largest singular value of the part of the mixed basis outside the FP64 span (rows are
        # orthonormal eigenvectors); this avoids the cancellation of arccos(sigma_min) near 1
        D = mixed_vecs - (mixed_vecs @ fp64_vecs.T) @ fp64_vecs
        sin_max = float(torch.sqrt(torch.clamp(torch.linalg.eigvalsh(D @ D.T).max(), min=0.0)).item())
        angle = float(np.arcsin(min(1.0, sin_max)))
        del D
    max_res_rel = float(np.max(res_mixed.residuals / np.maximum(np.abs(res_mixed.evals), 0.1)))

    # ---- end to end through the C ABI with host buffers (pinned), copies inside the timed region ----
    rp_h = torch.from_numpy(rp).pin_memory()
    ci_h = torch.from_numpy(ci).pin_memory()
    v_h = torch.from_numpy(v).pin_memory()
    v0_h = torch.from_numpy(start_host).pin_memory()
    ev_h = torch.empty((P.k, P.n), dtype=torch.float64).pin_memory()
    h2d = rp_h.numel() * 4 + ci_h.numel() * 4 + v_h.numel() * 8 + v0_h.numel() * 8
    d2h = ev_h.numel() * 8 + 2 * P.k * 8
    e2e_t = []
    for i in range(1 + args.e2e_steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        op_e = R.CsrOperator.from_host_pointers(ctx, P.n, ci.size, rp_h.data_ptr(), ci_h.data_ptr(),
                                                v_h.data_ptr())
        p = params("mixed")
        p.host_buffers = 1
        res_e = R.solve(ctx, op_e, p, v0=v0_h.data_ptr(), host=True, evecs_out=ev_h.data_ptr())
        op_e.close()
        torch.cuda.synchronize()
        if i > 0:
            e2e_t.append(time.perf_counter() - t0)
    e2e_value = replicas.job_rate(P.k, world, max_over_ranks(statistics.median(e2e_t)))
    assert np.array_equal(res_e.evals, res_mixed.evals)

    # ---- roofline of the dominant kernel: the fused filter degree-step (rm_step_kernel) ----
    # Algorithmic bytes of one degree-step over the n x s block: the matrix once (values + column
    # indices + row pointers) and three block passes (read x_{k-1}, read x_{k-2}, write x_k); the
    # correction filter's step (rm_step_src_kernel) also reads the residual block: four passes of
    # its storage type (bfloat16 or FP32, info.correction_element_bytes).
    # The step time is the CUDA-event time of the degree-step launches inside the timed solves
    # (info.time_filter_steps_ms, transposes excluded). Degree-1 filters (column-major path, at
    # most a few per solve) are counted in degree_steps but not timed, a < 0.1 % overstatement.
    nnz = ci.size
    b_a32 = nnz * (4 + 4) + (P.n + 1) * 4
    b_a64 = nnz * (8 + 4) + (P.n + 1) * 4
    bytes_fp32_step = b_a32 + 3 * P.n * s * 4
    ceb = int(infos[-1].get("correction_element_bytes", 4) or 4)
    bytes_corr_step = b_a32 + 4 * P.n * s * ceb
    bytes_fp64_step = b_a64 + 3 * P.n * s * 8
    # A correction filter of degree m launches m - 1 steps (e_1 = R comes from the residual kernel
    # of the Rayleigh-Ritz step), so its launches are its degree steps less its applications.
    f64steps = sum(i["fp64_degree_steps"] for i in infos)
    csteps_deg = sum(i["correction_degree_steps"] for i in infos)
    p32steps = sum(i["degree_steps"] for i in infos) - f64steps - csteps_deg
    csteps = csteps_deg - sum(i["correction_iterations"] for i in infos)
    fsteps = p32steps + csteps + f64steps
    tsteps = sum(i["time_filter_steps_ms"] for i in infos) * 1e-3
    alg_bytes = p32steps * bytes_fp32_step + csteps * bytes_corr_step + f64steps * bytes_fp64_step
    achieved = alg_bytes / tsteps / 1e9 if tsteps > 0 else None
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        peak, peak_src = float(peaks["hbm_gbs"]), "measured"
    except Exception:
        peak, peak_src = 6650.0, "fallback"
    # DRAM bytes per launch: the per-row figures of the ncu capture of the same kernel on the
    # 96^3 grid (profiles/), scaled to this block by its row count, mixed by precision like achieved
    traffic = None
    per_row = profile_dram_bytes_per_row()
    if per_row and fsteps:
        # without a capture of the correction step, its rows count as FP32 rows plus one more
        # block row (the residual block)
        corr_row = per_row.get("corr", per_row["fp32"] + s * ceb)
        traffic = P.n * (p32steps * per_row["fp32"] + csteps * corr_row + f64steps * per_row["fp64"]) / fsteps
    # ---- CPU baseline (rank 0, N = 1) ----
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            t_step, threads, kind = cpu_reference_sample(P, incr, buf, args.cpu_sample_degree, rp, ci, v)
            steps_solve = info64["degree_steps"] if info64 else CONFIG2_FP64_DEGREE_STEPS
            tts_cpu = t_step * steps_solve
            cpu = {"value": P.k / tts_cpu, "unit": "eigenpairs/s", "cores": threads, "kind": kind,
                   "sample": f"{args.cpu_sample_degree} degree-steps of the reference CPU filter on the full "
                             f"{s}-column block ({t_step * 1e3:.1f} ms/step) x {steps_solve} degree-steps of this "
                             f"run's FP64 solve; lower bound (excludes Lanczos, orthogonalisation, Rayleigh-Ritz)"}
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "eigenpairs/s", "cores": None, "kind": "reference",
                   "sample": f"unavailable: {e}"}

    value = replicas.job_rate(P.k, world, t_mixed * 1e-3)
    line = {
        "metric": METRIC, "value": value, "unit": "eigenpairs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_mixed, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 filter + f64", "data": "synthetic",
        "config": dict(config_dict(args, P.k, incr, buf, P.n, nnz), parallelism=f"replicas x{world}"),
        "tts_ms": {"mixed_p50": statistics.median(times), "mixed_p99": float(np.percentile(times, 99)),
                   "fp64_p50": statistics.median(t64) if t64 else None,
                   "fp64_p99": float(np.percentile(t64, 99)) if t64 else None},
        "fp64_eigenpairs_per_s": replicas.job_rate(P.k, world, t_fp64 * 1e-3) if t_fp64 else None,
        "speedup_mixed_vs_fp64": (t_fp64 / t_mixed) if t_fp64 else None,
        "accuracy": {"max_rel_eig_diff_mixed_vs_fp64": eig_err, "max_subspace_angle_mixed_vs_fp64": angle,
                     "max_rel_residual": max_res_rel, "found": int(res_mixed.info["found"])},
        "solve_info": {"mixed": {k2: infos[-1][k2] for k2 in ("inner_iterations", "degree_steps", "fp64_degree_steps",
                                                               "correction_iterations", "correction_degree_steps",
                                                               "mixed_iterations", "lanczos_iterations",
                                                               "cholqr_passes", "fused_rr", "fused_rr_fallbacks",
                                                               "time_lanczos_ms", "time_filter_ms",
                                                               "time_filter_steps_ms",
                                                               "time_ortho_ms", "time_eigenvalue_ms")},
                       "fp64": {k2: info64[k2] for k2 in ("inner_iterations", "degree_steps", "fp64_degree_steps",
                                                           "time_filter_ms",
                                                           "time_filter_steps_ms",
                                                           "time_ortho_ms", "time_eigenvalue_ms")} if info64 else None},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                     "peak_source": peak_src, "kernel": "rm_step_kernel + rm_step_src_kernel (fused filter degree-steps, CSR)",
                     "algorithmic_bytes_per_launch": alg_bytes / fsteps if fsteps else None,
                     "launches": fsteps, "fp64_launches": f64steps, "correction_launches": csteps,
                     "bytes_per_launch_fp32": bytes_fp32_step, "bytes_per_launch_correction": bytes_corr_step,
                     "bytes_per_launch_fp64": bytes_fp64_step},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": "eigenpairs/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(launches),
        "clocks": clk,
    }
    # ---- serving (configuration 4, the first --serve-count requests of the stream), N = 1 only ----
    if world == 1 and args.serve_count > 0:
        from rayleighchebyshevgpgpu_b200 import serve_bench
        try:
            sv = serve_bench.run(count=args.serve_count)
            line["serving"] = {k: sv[k] for k in ("requests", "completed", "eigenpairs_per_s", "requests_per_s",
                                                  "latency_ms_p50", "latency_ms_p99", "capacity_eigenpairs_per_s",
                                                  "arrival_rate_per_s", "max_active", "max_jobs_in_batch",
                                                  "hbm_peak_reserved_bytes")}
            line["serving"]["workload"] = (f"configuration-4 stream, first {args.serve_count} of 256 requests, "
                                           "Poisson arrivals at 0.8 x measured capacity, mixed precision")
        except Exception as e:  # reported, never required for the headline
            line["serving"] = {"unavailable": str(e)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    op.close()
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference_arm(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
