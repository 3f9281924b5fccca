"""Row sharding of the solve (rayleighchebyshevgpgpu_b200/sharding.py) on the CPU: the slab partition and
halo plan, and, on 2 and 3 gloo ranks, a sharded Chebyshev filter (halo exchange per degree step), a
sharded Gram matrix (all-reduce) and a whole sharded filter + Rayleigh-Ritz step (Gram and projection
all-reduces, replicated small eigensolve, residual norms by all-reduce) against one process. The
per-rank arithmetic here is numpy; on GPUs it is the library's kernels."""
import json
import os

import numpy as np
import pytest
import torch.multiprocessing as mp

from oracle import rc_oracle as O
from rayleighchebyshevgpgpu_b200 import problems
from rayleighchebyshevgpgpu_b200 import sharding as S

DIMS = (8, 6, 10)   # nx, ny, nz: z-slabs of nx*ny = 48 rows
S_COLS = 5
DEGREE = 7


def _problem():
    P = problems.small_laplacian(DIMS, seed=9, vmax=2.0, k=4)
    rp, ci, v = P.csr()
    return P, np.asarray(rp), np.asarray(ci), np.asarray(v)


def _block(n):
    return np.random.default_rng(4).standard_normal((n, S_COLS))


def test_partition_rows_whole_planes():
    r = S.partition_rows(480, 3, quantum=48)
    assert r == [(0, 192), (192, 336), (336, 480)]
    assert S.partition_rows(10, 4) == [(0, 3), (3, 6), (6, 8), (8, 10)]
    with pytest.raises(ValueError):
        S.partition_rows(480, 11, quantum=48)
    with pytest.raises(ValueError):
        S.partition_rows(100, 2, quantum=48)


def test_shard_plan_halos_are_neighbouring_planes():
    P, rp, ci, v = _problem()
    plan = S.shard_plan(rp, ci, S.partition_rows(P.n, 3, quantum=48))
    assert [(s.lo, s.hi) for s in plan] == [(0, 48), (48, 48), (48, 0)]
    assert [(s.send_down, s.send_up) for s in plan] == [(0, 48), (48, 48), (48, 0)]
    lrp, lci, lv = S.local_csr(rp, ci, v, plan[1])
    assert lrp[0] == 0 and lrp[-1] == lci.size == lv.size
    assert lci.min() >= 0 and lci.max() < plan[1].ext_rows


def test_shard_plan_rejects_couplings_beyond_the_neighbour():
    n = 12
    rows = [[i, (i + 7) % n] for i in range(n)]  # couples each row 7 rows away (wraps)
    rp = np.cumsum([0] + [len(r) for r in rows])
    ci = np.concatenate([sorted(r) for r in rows])
    with pytest.raises(ValueError):
        S.shard_plan(rp, ci, S.partition_rows(n, 3))


def _rank_main(rank: int, world: int, out_dir: str):
    import datetime

    import scipy.sparse as sp
    import torch
    import torch.distributed as dist

    # rendezvous through a file in the test's directory: no ports to collide
    dist.init_process_group("gloo", init_method="file://" + os.path.join(out_dir, "store"), rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        P, rp, ci, v = _problem()
        plan = S.shard_plan(rp, ci, S.partition_rows(P.n, world, quantum=DIMS[0] * DIMS[1]))
        sh = plan[rank]
        lrp, lci, lv = S.local_csr(rp, ci, v, sh)
        A_l = sp.csr_matrix((lv, lci, lrp), shape=(sh.rows, sh.ext_rows))
        X = _block(P.n)
        g1, g2 = O.gammas(DEGREE, 14.0, -0.5)
        own = slice(sh.lo, sh.lo + sh.rows)
        # x_k = g2 (g1 A x_{k-1} + x_{k-1}) - x_{k-2}, one halo exchange of x_{k-1} per step
        ext = torch.zeros((sh.ext_rows, S_COLS), dtype=torch.float64)
        ext[own] = torch.from_numpy(X[sh.r0:sh.r1])
        xkm2 = ext[own].clone()
        S.exchange_halo(ext, sh)
        xk = g2 * (g1 * torch.from_numpy(A_l @ ext.numpy()) + ext[own])
        for _k in range(2, DEGREE + 1):
            nxt = torch.zeros_like(ext)
            nxt[own] = xk
            S.exchange_halo(nxt, sh)
            y = g2 * (g1 * torch.from_numpy(A_l @ nxt.numpy()) + xk) - xkm2
            xkm2, xk = xk, y
        filt = (xk / (DEGREE + 1)).numpy()
        # Gram matrix of the filtered block: local product, summed over ranks
        G = torch.from_numpy(filt.T @ filt)
        S.allreduce_sum(G)
        dist.barrier()
    finally:
        dist.destroy_process_group()
    np.save(os.path.join(out_dir, f"filt{rank}.npy"), filt)
    np.save(os.path.join(out_dir, f"gram{rank}.npy"), G.numpy())
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"r0": sh.r0, "r1": sh.r1}, f)


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_filter_and_gram_match_the_oracle(tmp_path, world):
    mp.start_processes(_rank_main, args=(world, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    P, rp, ci, v = _problem()
    A = O.csr_matrix(rp, ci, v)
    g1, g2 = O.gammas(DEGREE, 14.0, -0.5)
    F = O.filter_block(A, _block(P.n), DEGREE, g1, g2)
    G = F.T @ F
    for r in range(world):
        rng = json.load(open(tmp_path / f"rank{r}.json"))
        filt = np.load(tmp_path / f"filt{r}.npy")
        np.testing.assert_allclose(filt, F[rng["r0"]:rng["r1"]], rtol=0, atol=1e-13 * np.abs(F).max())
        np.testing.assert_allclose(np.load(tmp_path / f"gram{r}.npy"), G, rtol=1e-12, atol=1e-12 * np.abs(G).max())


def _rr_single(A, X, m, g1, g2):
    """One filter + Rayleigh-Ritz step on one process: filtered block F, CholeskyQR basis, Ritz values
    and residual norms of the Ritz vectors."""
    F = O.filter_block(A, X, m, g1, g2)
    G = F.T @ F
    Lc = np.linalg.cholesky(G)
    T = np.linalg.inv(Lc).T                      # F T has orthonormal columns
    H = T.T @ (F.T @ (A @ F)) @ T
    lam, Q = np.linalg.eigh(0.5 * (H + H.T))
    Y = F @ (T @ Q)
    res = np.linalg.norm(A @ Y - Y * lam, axis=0)
    return lam, res


def _rr_rank_main(rank: int, world: int, out_dir: str):
    import datetime

    import scipy.sparse as sp
    import torch
    import torch.distributed as dist

    # rendezvous through a file in the test's directory: no ports to collide
    dist.init_process_group("gloo", init_method="file://" + os.path.join(out_dir, "store"), rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        P, rp, ci, v = _problem()
        plan = S.shard_plan(rp, ci, S.partition_rows(P.n, world, quantum=DIMS[0] * DIMS[1]))
        sh = plan[rank]
        lrp, lci, lv = S.local_csr(rp, ci, v, sh)
        A_l = sp.csr_matrix((lv, lci, lrp), shape=(sh.rows, sh.ext_rows))
        own = slice(sh.lo, sh.lo + sh.rows)

        def apply(x_own):  # A x on the own rows: one halo exchange, then the local product
            ext = torch.zeros((sh.ext_rows, x_own.shape[1]), dtype=torch.float64)
            ext[own] = torch.from_numpy(x_own)
            S.exchange_halo(ext, sh)
            return A_l @ ext.numpy()

        def allsum(a):
            return S.allreduce_sum(torch.from_numpy(np.ascontiguousarray(a))).numpy()

        g1, g2 = O.gammas(DEGREE, 14.0, -0.5)
        X = _block(P.n)[sh.r0:sh.r1]
        xkm2, xk = X, g2 * (g1 * apply(X) + X)
        for _k in range(2, DEGREE + 1):
            xkm2, xk = xk, g2 * (g1 * apply(xk) + xk) - xkm2
        F = xk / (DEGREE + 1)
        G = allsum(F.T @ F)                              # Gram: one all-reduce
        T = np.linalg.inv(np.linalg.cholesky(G)).T       # replicated small work
        AF = apply(F)
        H = T.T @ allsum(F.T @ AF) @ T                   # projection: one all-reduce
        lam, Q = np.linalg.eigh(0.5 * (H + H.T))         # replicated small eigensolve
        TQ = T @ Q
        Y, AY = F @ TQ, AF @ TQ
        res = np.sqrt(allsum(np.sum((AY - Y * lam) ** 2, axis=0)))  # residual norms: one all-reduce
        dist.barrier()
    finally:
        dist.destroy_process_group()
    np.save(os.path.join(out_dir, f"rr{rank}.npy"), np.stack([lam, res]))


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_rayleigh_ritz_step_matches_single_process(tmp_path, world):
    mp.start_processes(_rr_rank_main, args=(world, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    P, rp, ci, v = _problem()
    A = O.csr_matrix(rp, ci, v)
    g1, g2 = O.gammas(DEGREE, 14.0, -0.5)
    lam, res = _rr_single(A, _block(P.n), DEGREE, g1, g2)
    for r in range(world):
        got = np.load(tmp_path / f"rr{r}.npy")
        np.testing.assert_allclose(got[0], lam, rtol=1e-12, atol=1e-12)       # every rank, the same Ritz values
        np.testing.assert_allclose(got[1], res, rtol=1e-8, atol=1e-10 * np.abs(lam).max())


def test_extended_csr_is_square_with_empty_halo_rows():
    P, rp, ci, v = _problem()
    plan = S.shard_plan(rp, ci, S.partition_rows(P.n, 3, quantum=48))
    for sh in plan:
        erp, eci, ev = S.extended_csr(rp, ci, v, sh)
        assert erp.size == sh.ext_rows + 1 and erp[0] == 0 and erp[-1] == eci.size == ev.size
        assert np.all(np.diff(erp[:sh.lo + 1]) == 0) and np.all(np.diff(erp[sh.lo + sh.rows:]) == 0)
        assert eci.min() >= 0 and eci.max() < sh.ext_rows
        # the own rows of the extended operator times an extended block equal the global rows
        E = O.csr_matrix(erp, eci, ev)
        A = O.csr_matrix(rp, ci, v)
        x = _block(P.n)
        xe = x[sh.r0 - sh.lo:sh.r1 + sh.hi]
        np.testing.assert_array_equal((E @ xe)[sh.lo:sh.lo + sh.rows], (A @ x)[sh.r0:sh.r1])
