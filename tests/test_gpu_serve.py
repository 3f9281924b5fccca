"""The request server (rc_server_*, rc_serve_*) on the GPU: every served result is the same as
the solve run alone and as rc_solve, whatever else shares its batches; admission keeps the
device footprint under the HBM budget; cancellation and teardown never hang."""
import time

import numpy as np
import pytest

from oracle import rc_oracle as O
from rayleighchebyshevgpgpu_b200 import problems
from rayleighchebyshevgpgpu_b200 import runtime as R

pytestmark = pytest.mark.gpu


def _mix():
    """Small requests of every served form: 2D 5-point and 3D 7-point stencils, a CSR operator,
    different k, tolerances and precisions."""
    reqs = []
    for i, (dims, k, tol, prec, form) in enumerate([
        ((48, 40), 8, 1e-10, "mixed", "stencil"),
        ((14, 12, 11), 16, 1e-10, "mixed", "stencil"),
        ((64, 50), 16, 1e-8, "mixed", "csr"),
        ((12, 12, 12), 8, 1e-10, "fp64", "stencil"),
        ((30, 30), 32, 1e-10, "mixed", "stencil"),
        ((10, 11, 13), 8, 1e-8, "fp64", "csr"),
    ]):
        P = problems.small_laplacian(dims, seed=20 + i, vmax=3.0, k=k)
        P.tol = tol
        reqs.append((P, prec, form))
    return reqs


def _done(h, timeout_ms):
    """Wait for a request; a request that did not finish raises with its own status and message."""
    st = h.wait(timeout_ms)
    if st != "done":
        h.result()
    assert st == "done", st


def _params(P, prec, seed):
    p = R.make_params(P.k, P.tol, precision=prec, stop="RESIDUAL_ONLY")
    p.seed = seed
    return p


def _start(P):
    incr, buf = problems.block_sizes(P.k)
    return P.start_block(incr + buf)


def test_served_results_equal_alone_in_mix_and_solo(ctx):
    reqs = _mix()
    ops = [R.operator_from_problem(ctx, P, form) for P, _, form in reqs]
    # rc_solve, one at a time
    solo = [R.solve(ctx, op, _params(P, prec, 7 + i), v0=_start(P), host=True)
            for i, ((P, prec, _), op) in enumerate(zip(reqs, ops))]
    # served alone: one request in the server at a time
    with R.Server(0, max_active=4) as srv:
        alone = []
        for i, ((P, prec, _), op) in enumerate(zip(reqs, ops)):
            rq = srv.submit(op, _params(P, prec, 7 + i), v0=_start(P))
            _done(rq, 120000)
            alone.append(rq.result())
        st_alone = srv.stats()
    # served in the mix: everything submitted at once
    with R.Server(0, max_active=8) as srv:
        handles = [srv.submit(op, _params(P, prec, 7 + i), v0=_start(P))
                   for i, ((P, prec, _), op) in enumerate(zip(reqs, ops))]
        mixed = []
        for h in handles:
            _done(h, 120000)
            mixed.append(h.result())
        st_mix = srv.stats()
    assert st_alone["max_jobs_in_batch"] == 1
    assert st_mix["max_jobs_in_batch"] >= 2, st_mix
    assert st_mix["batches"] < st_mix["batched_jobs"]
    for (P, prec, form), s, a, m in zip(reqs, solo, alone, mixed):
        assert a.info["found"] == P.k and m.info["found"] == P.k
        # a batch computes each solve exactly as alone
        assert np.array_equal(a.evals, m.evals), (P.name, a.evals - m.evals)
        assert np.array_equal(a.residuals, m.residuals)
        assert np.array_equal(a.evecs, m.evecs)
        np.testing.assert_allclose(m.evals, s.evals, rtol=1e-12)
        A = O.csr_matrix(*P.csr())
        dense = O.dense_lowest(A, P.k)
        np.testing.assert_allclose(m.evals, dense, rtol=max(10 * P.tol, 1e-10), atol=1e-12)
        X = m.evecs.T
        r = np.linalg.norm(A @ X - X * m.evals, axis=0) / np.maximum(np.abs(m.evals), 0.1)
        assert r.max() <= 1.5 * P.tol, (P.name, r.max())
        assert m.info["request"]["batches"] > 0
    for op in ops:
        op.close()


def test_graphs_and_direct_launches_agree(ctx):
    reqs = _mix()[:3]
    ops = [R.operator_from_problem(ctx, P, form) for P, _, form in reqs]
    out = {}
    for graphs in (True, False):
        with R.Server(0, max_active=4, use_graphs=graphs) as srv:
            hs = [srv.submit(op, _params(P, prec, 3 + i), v0=_start(P))
                  for i, ((P, prec, _), op) in enumerate(zip(reqs, ops))]
            states = [h.wait(120000) for h in hs]
            # result() raises with the request's own status and message when it failed
            out[graphs] = [h.result() for h in hs]
            assert states == ["done"] * len(hs)
            st = srv.stats()
            if graphs:
                assert st["graph_launches"] == st["batches"] and st["graphs_built"] >= 1
            else:
                assert st["graph_launches"] == 0
    for a, b in zip(out[True], out[False]):
        assert np.array_equal(a.evals, b.evals)
    for op in ops:
        op.close()


def test_admission_keeps_footprint_under_budget(ctx):
    Ps = [problems.small_laplacian((40, 40, 40), seed=40 + i, vmax=2.0, k=16) for i in range(6)]
    ops = [R.StencilOperator(ctx, 7, P.dims, P.diag, P.offdiag) for P in Ps]
    # budget: room for about two of these solves at once (each ~ 64000 * (4*24 + 16) * 8 B + slack)
    with R.Server(0, max_active=6) as probe:
        one = probe.submit(ops[0], _params(Ps[0], "mixed", 1))
        _done(one, 120000)
        need = one.info()["reserved_bytes"]
    budget = int(2.5 * (need + Ps[0].n * 8 * 2))
    with R.Server(0, max_active=6, budget_bytes=budget) as srv:
        hs = [srv.submit(op, _params(P, "mixed", 11 + i)) for i, (P, op) in enumerate(zip(Ps, ops))]
        for h in hs:
            _done(h, 180000)
        st = srv.stats()
        assert st["completed"] == 6
        assert st["bytes_peak"] <= budget
        assert st["bytes_in_use"] == 0
        for h in hs:
            inf = h.info()
            assert 0 < inf["device_bytes"] <= inf["reserved_bytes"], inf
        # with room for two solves, some request had to wait for memory
        assert max(h.info()["queue_ms"] for h in hs) > 0.0
    for op in ops:
        op.close()


def test_request_above_budget_is_rejected(ctx):
    P = problems.small_laplacian((32, 32, 32), seed=3, k=16)
    op = R.StencilOperator(ctx, 7, P.dims, P.diag, P.offdiag)
    with R.Server(0, max_active=2, budget_bytes=1 << 20) as srv:
        with pytest.raises(R.capi.RCError) as e:
            srv.submit(op, _params(P, "mixed", 1))
        assert e.value.status == 3  # RC_ERR_NOMEM
    op.close()


def test_cancel_queued_and_running(ctx):
    big = problems.small_laplacian((96, 96, 48), seed=5, vmax=4.0, k=64)
    small = problems.small_laplacian((20, 20), seed=6, k=8)
    opb = R.StencilOperator(ctx, 7, big.dims, big.diag, big.offdiag)
    ops = R.StencilOperator(ctx, 5, small.dims, small.diag, small.offdiag)
    with R.Server(0, max_active=1) as srv:
        hb = srv.submit(opb, _params(big, "fp64", 1))
        hs = srv.submit(ops, _params(small, "mixed", 2))
        assert hs.state() == "queued"
        hs.cancel()
        assert hs.state() == "cancelled"
        t0 = time.time()
        while hb.state() == "queued" and time.time() - t0 < 60:
            time.sleep(0.01)
        hb.cancel()
        assert hb.wait(120000) in ("cancelled", "done")
        st = srv.stats()
        assert st["cancelled"] >= 1
        # the server keeps serving after cancellations
        again = srv.submit(ops, _params(small, "mixed", 2))
        _done(again, 120000)
        assert again.result().info["found"] == small.k
    opb.close()
    ops.close()


def test_callback_operator_is_served_unbatched(ctx):
    """A foreign apply(in, out, alpha, beta) operator runs on the single-solve path inside its slot
    (the batched kernels need the operator's structure) and still gives the LAPACK eigenvalues."""
    import torch
    P = problems.small_laplacian((18, 17), seed=13)
    rp, ci, v = P.csr()
    A = O.csr_matrix(rp, ci, v)
    At = torch.sparse_csr_tensor(torch.from_numpy(rp.astype(np.int64)), torch.from_numpy(ci.astype(np.int64)),
                                 torch.from_numpy(v), size=(P.n, P.n)).cuda()
    calls = {"n": 0}

    def apply(pin, pout, n, s, ld, alpha, beta, stream):
        calls["n"] += 1
        torch.cuda.synchronize()
        src = _wrap(pin, n, s)
        dst = _wrap(pout, n, s)
        y = torch.sparse.mm(At, src.T).T
        dst.copy_(alpha.real * y + beta.real * dst)
        torch.cuda.synchronize()
        return 0

    op = R.CallbackOperator(ctx, P.n, apply)
    with R.Server(0, max_active=2) as srv:
        h = srv.submit(op, _params(P, "fp64", 4), v0=_start(P))
        _done(h, 120000)
        res = h.result()
        st = srv.stats()
    assert calls["n"] > 10 and st["batched_jobs"] == 0
    np.testing.assert_allclose(res.evals, O.dense_lowest(A, P.k), rtol=1e-10)
    op.close()


def _wrap(ptr, n, s):
    """View a device pointer as an (s, n) float64 CUDA tensor (column-major n x s block)."""
    import torch

    class _CAI:
        def __init__(self):
            self.__cuda_array_interface__ = {"shape": (s, n), "typestr": "<f8", "data": (ptr, False), "version": 3,
                                             "strides": None}
    return torch.as_tensor(_CAI(), device="cuda")


def test_destroy_with_queued_requests_does_not_hang(ctx):
    P = problems.small_laplacian((64, 64, 32), seed=9, vmax=4.0, k=32)
    op = R.StencilOperator(ctx, 7, P.dims, P.diag, P.offdiag)
    srv = R.Server(0, max_active=1)
    hs = [srv.submit(op, _params(P, "mixed", i)) for i in range(4)]
    t0 = time.time()
    srv.close()
    assert time.time() - t0 < 120
    op.close()
    del hs
