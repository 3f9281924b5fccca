"""Benchmark: time-to-solution and eigenpairs/s at residual <= 1e-10 on one B200, mixed vs FP64.

Workload (configuration 2): lowest 64 eigenpairs of the 3D 7-point Dirichlet Laplacian on 128^3
(n = 2,097,152; CSR with FP64 values and int32 indices, 14,581,760 nnz) plus a U[0,4) potential
(seed 2); start block N(0,1) (seed 3), subspace 64 + 32 buffer; stop test RESIDUAL_ONLY at 1e-10.
A "step" is one whole solve (Lanczos bounds, then filtered subspace iteration with Rayleigh-Ritz
until every residual <= 1e-10) from the operator and start block resident in HBM to eigenvalues
and residuals on the host. MIXED: the first filter application in FP32, every later one as the
correction filter (bfloat16 storage, FP32 arithmetic); everything else FP64.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--side 128]

--impl reference times the reference's own CPU solver (built from its sources into oracle/_ref) on
the same workload: each step is one bounded sample (one inner iteration of its solve), and the
reported time-to-solution is an estimate from those samples and the iteration counts of the
reference's own full solve of this workload (tests/golden/config2_solve.json).

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
# The reference's own CPU solve of the benchmark workload (RayleighChebyshevLM::getMinEigenSystem built
# from its sources, run once to completion by tests/golden/make_golden_large.py): eigenvalues for the
# parity check and the reference's own iteration and operator-apply counts for the CPU time estimate.
REF_SOLVE_FIXTURE = os.path.join(ROOT, "tests", "golden", "config2_solve.json")
DTYPE = "f64 (Rayleigh-Ritz, orthonormalisation, residuals); filter: bf16 storage with f32 arithmetic"


def reference_solve_fixture(side: int):
    try:
        g = json.load(open(REF_SOLVE_FIXTURE))
    except (OSError, ValueError):
        return None
    return g if g.get("side") == side else None


def reference_counts(g) -> dict | None:
    """Inner iterations and filter degree-steps of the reference's own solve, from its counters
    (RayleighChebyshevLM.h:1224-1294): every inner iteration adds starDegree*s (filter), s
    (formVtAV) and residualCheckCount (= incr on a single outer pass) to OpApply, and one to
    'eigenvalue'."""
    if not g:
        return None
    s = g["incr"] + g["buffer"]
    iters = int(g["count_eigenvalue"])
    steps = (int(g["count_opapply"]) - iters * (s + g["incr"])) // s
    return {"inner_iterations": iters, "degree_steps": steps}


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
    ap.add_argument("--cpu-sample-degree", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serve-count", type=int, default=64,
                    help="requests of the configuration-4 serving stream run after the timed solves (0: skip)")
    ap.add_argument("--other-configs", default="3,5",
                    help="configurations solved once each in mixed precision and in FP64 after the headline, "
                         "reported under other_workloads (empty: skip)")
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


def config_dict(args, k, incr, buf, n, nnz, world=1):
    return {"workload": f"config2: 3D 7-point Laplacian {args.side}^3 + U[0,4) potential, CSR fp64/int32, "
                        f"lowest {k} eigenpairs, tol 1e-10 RESIDUAL_ONLY",
            "n": n, "nnz": nnz, "k": k, "subspace": incr + buf, "increment": incr, "buffer": buf,
            "operator_form": "csr", "start_block": "N(0,1) seed 3",
            "l2": "inputs larger than L2 (start block 1.6 GB, operator 183 MB)",
            "parallelism": f"replicas x{world}"}


# ---------------------------------------------------------------------------------------------
# CPU baseline: the reference's own CPU solver (RayleighChebyshevLM, built from its sources into
# oracle/_ref) on the full benchmark block, all host threads. One inner iteration of its solve has
# three phases: the filter (LanczosCpolyOperatorLM::apply, timed per degree-step), one modified
# Gram-Schmidt orthogonalisation, and one Rayleigh-Ritz step (formVtAV, Jacobi,
# createEigenVectorsAndResiduals). A sample times one phase; the phases rotate over the samples.
# The time-to-solution estimate is
#   filter seconds per degree-step x the reference solve's degree-steps
#   + (orthogonalisation + Rayleigh-Ritz seconds) x its inner iterations,
# with both counts from the reference's own full solve of this workload (tests/golden).
# ---------------------------------------------------------------------------------------------
PHASES = ("filter", "ortho", "rr")


class ReferenceSampler:
    def __init__(self, P, incr, buf, rp, ci, v, degree):
        from oracle import ref_io
        self.ref_io = ref_io
        self.P, self.incr, self.buf, self.degree = P, incr, buf, degree
        self.s = incr + buf
        self.threads = os.cpu_count() or 1
        self.kind = "reference" if ref_io.ref_available() else "port"
        g = reference_solve_fixture(round(P.n ** (1 / 3)))
        self.lmin = g["min_eig_est"] if g else 0.4
        self.lmax = g["max_eig_est"] if g else 16.0
        self.dir = tempfile.mkdtemp()
        self.path = os.path.join(self.dir, "c2.bin")
        if self.kind == "reference":
            ref_io.write_problem(self.path, rp, ci, v, P.start_block(self.s))
        else:
            from oracle import rc_oracle as O
            self.A = O.csr_matrix(rp, ci, v)
            self.X = P.start_block(self.s).T.copy()

    def sample(self, phase: str) -> dict:
        """Seconds of one phase of one inner iteration ("filter": per degree-step)."""
        if self.kind == "reference":
            r = self.ref_io.run_ref("phases", self.path, degree=self.degree, bound=self.lmax, shift=-self.lmin,
                                    rescheck=self.incr, threads=self.threads, do=phase)
            sec = {"filter": r["filter_seconds"] / self.degree, "ortho": r["ortho_seconds"],
                   "rr": r["rr_seconds"]}[phase]
            return {"phase": phase, "seconds": sec, "wall": sec * (self.degree if phase == "filter" else 1),
                    "threads": r["threads"]}
        # oracle port: numpy/scipy, the same three phases
        from oracle import rc_oracle as O
        t0 = time.perf_counter()
        if phase == "filter":
            g1, g2 = O.gammas(self.degree, self.lmax, -self.lmin)
            O.filter_block(self.A, self.X, self.degree, g1, g2)
        elif phase == "ortho":
            np.linalg.qr(self.X)
        else:
            W = self.A @ self.X
            lam, Q = np.linalg.eigh(self.X.T @ W)
            Y = self.X @ Q
            np.linalg.norm(self.A @ Y[:, :self.incr] - Y[:, :self.incr] * lam[:self.incr], axis=0)
        t = time.perf_counter() - t0
        return {"phase": phase, "seconds": t / (self.degree if phase == "filter" else 1), "wall": t, "threads": 1}

    def estimate(self, samples: list, counts: dict) -> dict:
        med = {ph: statistics.median([x["seconds"] for x in samples if x["phase"] == ph]) for ph in PHASES}
        tts = med["filter"] * counts["degree_steps"] + (med["ortho"] + med["rr"]) * counts["inner_iterations"]
        return {"tts_s": tts, "filter_step_s": med["filter"], "ortho_s": med["ortho"], "rr_s": med["rr"]}

    def close(self):
        try:
            os.remove(self.path)
        except OSError:
            pass


def describe_estimate(kind, threads, degree, s, est, counts, g):
    meas = (f"; the reference's full solve of this workload, run to completion once on {g['reference_threads']} "
            f"threads of the build machine, took {g['reference_seconds']:.0f} s") if g else ""
    return (f"estimate: the phases of one inner iteration of the reference CPU solver ({kind}, {threads} threads) "
            f"on the full {s}-column block, one phase per sample in rotation ({degree} filter degree-steps, "
            f"{est['filter_step_s'] * 1e3:.0f} ms each; orthogonalisation {est['ortho_s'] * 1e3:.0f} ms; "
            f"Rayleigh-Ritz {est['rr_s'] * 1e3:.0f} ms); "
            f"time-to-solution = filter time per degree-step x {counts['degree_steps']} degree-steps + "
            f"(orthogonalisation + Rayleigh-Ritz) x {counts['inner_iterations']} inner iterations, the counts of "
            f"the reference's own solve (excludes its Lanczos bounds){meas}")


def reference_counts_or_default(side):
    counts = reference_counts(reference_solve_fixture(side))
    # without the fixture (another grid side): this library's FP64 solve of configuration 2 took
    # 116 inner iterations and 1659 degree-steps
    return counts or {"inner_iterations": 116, "degree_steps": 1659}


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    from rayleighchebyshevgpgpu_b200 import problems
    P = problems.config2(args.side)
    incr, buf = problems.block_sizes(P.k)
    rp, ci, v = P.csr()
    sampler = ReferenceSampler(P, incr, buf, rp, ci, v, args.cpu_sample_degree)
    samples, wall = [], []
    # warm-up samples rotate from the filter; timed samples cover every phase at least once
    for i in range(args.warmup + max(args.steps, len(PHASES))):
        ph = PHASES[(i - args.warmup) % len(PHASES)] if i >= args.warmup else PHASES[i % len(PHASES)]
        x = sampler.sample(ph)
        if i >= args.warmup:
            samples.append(x)
            wall.append(x["wall"])
    sampler.close()
    g = reference_solve_fixture(args.side)
    counts = reference_counts_or_default(args.side)
    est = sampler.estimate(samples, counts)
    value = P.k / est["tts_s"]
    threads = samples[-1]["threads"]
    desc = describe_estimate(sampler.kind, threads, args.cpu_sample_degree, incr + buf, est, counts, g)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "eigenpairs/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": statistics.fmean(wall) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_dict(args, P.k, incr, buf, P.n, len(ci), world),
        "estimate": True,
        "estimate_rule": "tts = filter_s_per_degree_step * reference_degree_steps + (ortho_s + rr_s) * "
                         "reference_inner_iterations (medians over the samples); a step is one timed sample of "
                         "one phase of an inner iteration, phases in rotation",
        "reference_tts_s": est["tts_s"],
        "cpu_baseline": {"value": value, "unit": "eigenpairs/s", "cores": threads, "kind": sampler.kind,
                         "sample": desc},
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
    # residuals recomputed outside the library: torch's own sparse CSR product in FP64 on the returned
    # eigenvectors (rows of the k x n blocks), relative to max(|lambda|, 0.1) as the stop test
    with torch.no_grad():
        A_t = torch.sparse_csr_tensor(torch.from_numpy(rp.astype(np.int64)), torch.from_numpy(ci.astype(np.int64)),
                                      torch.from_numpy(v), size=(P.n, P.n), dtype=torch.float64, device="cuda")
        indep = {}
        for name, vecs, evals in (("mixed", mixed_vecs, res_mixed.evals), ("fp64", fp64_vecs, res64.evals)):
            AX = torch.sparse.mm(A_t, vecs.T.contiguous())
            lam_t = torch.from_numpy(evals).cuda()
            rn = torch.linalg.vector_norm(AX - vecs.T * lam_t, dim=0).cpu().numpy()
            indep[name] = float(np.max(rn / np.maximum(np.abs(evals), 0.1)))
            del AX
        del A_t
    # parity with the reference's own CPU solve of this workload (tests/golden fixture)
    gref = reference_solve_fixture(args.side)
    parity = None
    if gref:
        ev_ref = np.asarray(gref["eigenvalues"])
        parity = {"reference": "RayleighChebyshevLM CPU solve, same operator, start block, block sizes, stop test",
                  "max_rel_eig_err_mixed": float(np.max(np.abs(res_mixed.evals - ev_ref) / np.abs(ev_ref))),
                  "max_rel_eig_err_fp64": float(np.max(np.abs(res64.evals - ev_ref) / np.abs(ev_ref)))}

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
    # ---- CPU baseline (rank 0, N = 1): two samples of the reference's own CPU solver ----
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            sampler = ReferenceSampler(P, incr, buf, rp, ci, v, args.cpu_sample_degree)
            samples = [sampler.sample(ph) for ph in PHASES]
            sampler.close()
            counts = reference_counts_or_default(args.side)
            est = sampler.estimate(samples, counts)
            cpu = {"value": P.k / est["tts_s"], "unit": "eigenpairs/s", "cores": samples[-1]["threads"],
                   "kind": sampler.kind,
                   "sample": describe_estimate(sampler.kind, samples[-1]["threads"], args.cpu_sample_degree, s, est,
                                               counts, reference_solve_fixture(args.side))}
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "eigenpairs/s", "cores": None, "kind": "reference",
                   "sample": f"unavailable: {e}"}

    value = replicas.job_rate(P.k, world, t_mixed * 1e-3)
    line = {
        "metric": METRIC, "value": value, "unit": "eigenpairs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_mixed, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": DTYPE, "data": "synthetic",
        "config": config_dict(args, P.k, incr, buf, P.n, nnz, world),
        "tts_ms": {"mixed_p50": statistics.median(times), "mixed_p99": float(np.percentile(times, 99)),
                   "fp64_p50": statistics.median(t64) if t64 else None,
                   "fp64_p99": float(np.percentile(t64, 99)) if t64 else None},
        "fp64_eigenpairs_per_s": replicas.job_rate(P.k, world, t_fp64 * 1e-3) if t_fp64 else None,
        "speedup_mixed_vs_fp64": (t_fp64 / t_mixed) if t_fp64 else None,
        "accuracy": {"max_rel_eig_diff_mixed_vs_fp64": eig_err, "max_subspace_angle_mixed_vs_fp64": angle,
                     "max_rel_residual": max_res_rel,
                     "max_rel_residual_independent": indep,
                     "vs_reference_solve": parity, "found": int(res_mixed.info["found"])},
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
    # ---- configurations 3 and 5, one mixed and one FP64 solve each, N = 1 only ----
    if world == 1 and args.other_configs:
        others = {}
        for c in [int(x) for x in args.other_configs.split(",") if x.strip()]:
            try:
                others[f"config{c}"] = other_workload(c, ctx, stream)
            except Exception as e:  # reported, never required for the headline
                others[f"config{c}"] = {"unavailable": str(e)}
        line["other_workloads"] = others
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


OTHER_NAMES = {
    3: "config3: 3D tight-binding 96^3, Peierls flux 1/17 on y-bonds, U[-1,1) potential, complex Hermitian "
       "7-point stencil, lowest 128 eigenpairs, tol 1e-9 RESIDUAL_ONLY",
    5: "config5: 3D 27-point stencil 256^3, off-diagonal -1/26, diagonal 1 + U[0,2) potential, lowest 32 "
       "eigenpairs, tol 1e-10 RESIDUAL_ONLY",
}


def other_workload(config: int, ctx, stream) -> dict:
    """One configuration beside the headline: a warm-up solve, then one mixed and one FP64 solve from
    the same start block (CUDA events on the solver stream), the eigenvalues of the two compared, and
    every residual recomputed with the stencil written out in plain torch (verify.stencil_residuals)."""
    import torch

    from rayleighchebyshevgpgpu_b200 import problems
    from rayleighchebyshevgpgpu_b200 import runtime as R
    from rayleighchebyshevgpgpu_b200.verify import stencil_residuals

    P = problems.config3() if config == 3 else problems.config5()
    incr, buf = problems.block_sizes(P.k)
    s = incr + buf
    op = R.operator_from_problem(ctx, P, "stencil")
    v0 = torch.from_numpy(P.start_block(s)).cuda()
    evecs = torch.empty((P.k, P.n), dtype=v0.dtype, device="cuda")

    def run(prec, iters=0):
        p = R.make_params(P.k, P.tol, incr=incr, buffer=buf, precision=prec, stop="RESIDUAL_ONLY", phase_timing=1)
        p.v0_cols = s
        if iters:
            p.max_inner_loop = iters
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        res = R.solve(ctx, op, p, v0=v0, host=False, evecs_out=evecs)
        e1.record(stream)
        torch.cuda.synchronize()
        return res, e0.elapsed_time(e1)

    run("mixed", iters=4)  # warm-up: operator copies, scratch slots, kernel modules
    out = {"workload": OTHER_NAMES[config], "n": P.n, "k": P.k, "subspace": s, "operator_form": "stencil",
           "start_block": f"N(0,1) seed {P.start_seed}"}
    solves = {}
    for prec in ("mixed", "fp64"):
        res, ms = run(prec)
        rel = stencil_residuals(P, evecs[:P.k], res.evals)
        info = res.info
        solves[prec] = (res, ms)
        out[prec] = {"tts_ms": ms, "eigenpairs_per_s": P.k / (ms * 1e-3), "found": int(info["found"]),
                     "max_rel_residual_independent": float(rel.max()),
                     "solve_info": {k: info[k] for k in ("inner_iterations", "degree_steps", "fp64_degree_steps",
                                                         "correction_iterations", "time_filter_ms",
                                                         "time_eigenvalue_ms", "time_ortho_ms", "time_lanczos_ms")}}
    (rm, tm), (r64, t64) = solves["mixed"], solves["fp64"]
    out["speedup_mixed_vs_fp64"] = t64 / tm
    out["max_rel_eig_diff_mixed_vs_fp64"] = float(np.max(np.abs(rm.evals - r64.evals) / np.abs(r64.evals)))
    del v0, evecs
    op.close()
    torch.cuda.empty_cache()
    return out


def main():
    args = parse()
    if args.impl == "reference":
        run_reference_arm(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
