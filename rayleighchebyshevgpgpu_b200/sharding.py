"""Row sharding of the Rayleigh-Chebyshev solve over ranks: the host-side plan and collectives.

A sharded solve splits the n rows of the operator and of every n x s block into contiguous slabs, one
per rank (whole z-planes for stencil orderings, so a halo is whole planes). Per filter degree-step a
rank needs the rows of x_{k-1} that its own rows couple to and that other ranks own: for a banded
operator these are the `lo` rows just below its slab and the `hi` rows just above it, held by its two
neighbours. In the row-major block layout of the filter those halos are contiguous runs of rows, so
the exchange is one send and one receive per neighbour and direction. Per Rayleigh-Ritz or
CholeskyQR step the s x s Gram matrices are summed over ranks (all-reduce), and the small
eigensolve is repeated on every rank.

This module holds that plan and the two collectives over torch.distributed (NCCL between GPUs, gloo
on the CPU):
  partition_rows   the slab partition;
  shard_plan       each rank's rows, halo extent and neighbours' halo needs, from the CSR pattern;
  local_csr        the rank's rows with columns rebased to its extended block [halo_lo | own | halo_hi];
  exchange_halo    fills the halo rows of an extended row-major block from the neighbours;
  allreduce_sum    sums a Gram matrix (or any tensor) over ranks;
  extended_csr     the rank's operator on its whole extended block, halo rows empty: with it, one
                   unsharded row-major degree step over the extended block computes the rank's rows
                   (the halo rows of the result are discarded and refilled by the next exchange).
and the device side of the sharded filter:
  rank_operator    the rank's operator on its extended block on the GPU (extended CSR, or the stencil
                   on the sub-grid of its planes plus halo planes);
  extended_rows    a rank's extended row-major block cut from a global one;
  sharded_filter   the Chebyshev filter on a rank's extended block: one library degree step
                   (rc_filter_step_rm) per degree, the halo exchange between steps. Each rank's own
                   rows come out bit for bit as the unsharded filter computes them.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Sequence, Tuple

import numpy as np


def partition_rows(n: int, world: int, quantum: int = 1) -> List[Tuple[int, int]]:
    """Contiguous row ranges [r0, r1) of the ranks: whole quanta (e.g. nx*ny rows, one z-plane),
    counts differing by at most one quantum, every rank non-empty."""
    if n % quantum != 0:
        raise ValueError("n is not a multiple of the quantum")
    q = n // quantum
    if world < 1 or world > q:
        raise ValueError(f"cannot split {q} quanta over {world} ranks")
    base, extra = divmod(q, world)
    out, r = [], 0
    for k in range(world):
        cnt = (base + (1 if k < extra else 0)) * quantum
        out.append((r, r + cnt))
        r += cnt
    return out


@dataclass(frozen=True)
class Shard:
    rank: int
    world: int
    r0: int          # own rows [r0, r1)
    r1: int
    lo: int          # halo rows below: [r0 - lo, r0), owned by rank - 1
    hi: int          # halo rows above: [r1, r1 + hi), owned by rank + 1
    send_down: int   # own first rows rank - 1 needs (its hi)
    send_up: int     # own last rows rank + 1 needs (its lo)

    @property
    def rows(self) -> int:
        return self.r1 - self.r0

    @property
    def ext_rows(self) -> int:
        return self.lo + self.rows + self.hi


def _halo(rowptr: np.ndarray, colind: np.ndarray, r0: int, r1: int) -> Tuple[int, int]:
    cols = colind[rowptr[r0]:rowptr[r1]]
    if cols.size == 0:
        return 0, 0
    return max(0, r0 - int(cols.min())), max(0, int(cols.max()) + 1 - r1)


def shard_plan(rowptr: Sequence[int], colind: Sequence[int], ranges: List[Tuple[int, int]]) -> List[Shard]:
    """Each rank's halo extent from the CSR pattern. A halo must lie within the neighbouring rank's
    rows (nearest-neighbour exchange): a coupling that reaches further raises ValueError."""
    rp = np.asarray(rowptr, dtype=np.int64)
    ci = np.asarray(colind, dtype=np.int64)
    world = len(ranges)
    halos = [_halo(rp, ci, r0, r1) for r0, r1 in ranges]
    out = []
    for k, ((r0, r1), (lo, hi)) in enumerate(zip(ranges, halos)):
        if lo and (k == 0 or lo > ranges[k - 1][1] - ranges[k - 1][0]):
            raise ValueError(f"rank {k}: rows couple below the neighbouring slab")
        if hi and (k == world - 1 or hi > ranges[k + 1][1] - ranges[k + 1][0]):
            raise ValueError(f"rank {k}: rows couple above the neighbouring slab")
        send_down = halos[k - 1][1] if k > 0 else 0
        send_up = halos[k + 1][0] if k + 1 < world else 0
        out.append(Shard(k, world, r0, r1, lo, hi, send_down, send_up))
    return out


def local_csr(rowptr, colind, vals, sh: Shard):
    """The rank's rows, columns rebased to the extended block (column j -> j - (r0 - lo)); the order
    of the entries within a row is kept, so a row's products sum in the same order as unsharded."""
    rp = np.asarray(rowptr, dtype=np.int64)
    a, b = int(rp[sh.r0]), int(rp[sh.r1])
    lrp = (rp[sh.r0:sh.r1 + 1] - a).astype(np.int32)
    lci = (np.asarray(colind[a:b], dtype=np.int64) - (sh.r0 - sh.lo)).astype(np.int32)
    return lrp, lci, np.asarray(vals[a:b])


def exchange_halo(x_ext, sh: Shard, group=None) -> None:
    """Fill the halo rows of the extended row-major block x_ext (ext_rows x ld, own rows at
    [lo, lo + rows)) from the neighbours, in place. Every rank calls it at the same step."""
    import torch.distributed as dist

    ops = []
    own0 = sh.lo
    if sh.send_down:
        ops.append(dist.P2POp(dist.isend, x_ext[own0:own0 + sh.send_down].contiguous(), sh.rank - 1, group))
    if sh.send_up:
        ops.append(dist.P2POp(dist.isend, x_ext[own0 + sh.rows - sh.send_up:own0 + sh.rows].contiguous(),
                              sh.rank + 1, group))
    recv = []
    if sh.lo:
        buf = x_ext.new_empty((sh.lo,) + tuple(x_ext.shape[1:]))
        ops.append(dist.P2POp(dist.irecv, buf, sh.rank - 1, group))
        recv.append((0, buf))
    if sh.hi:
        buf = x_ext.new_empty((sh.hi,) + tuple(x_ext.shape[1:]))
        ops.append(dist.P2POp(dist.irecv, buf, sh.rank + 1, group))
        recv.append((own0 + sh.rows, buf))
    if ops:
        for w in dist.batch_isend_irecv(ops):
            w.wait()
    for at, buf in recv:
        x_ext[at:at + buf.shape[0]] = buf


def allreduce_sum(t, group=None):
    """Sum a tensor over ranks in place (the Gram matrices of a Rayleigh-Ritz step)."""
    import torch.distributed as dist

    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t


def extended_csr(rowptr, colind, vals, sh: Shard):
    """The rank's operator as a square CSR matrix on its extended block (ext_rows rows): its own rows
    at [lo, lo + rows) with columns in the extended numbering, the halo rows empty."""
    lrp, lci, lv = local_csr(rowptr, colind, vals, sh)
    rp = np.concatenate([np.zeros(sh.lo, dtype=np.int32), lrp, np.full(sh.hi, lrp[-1], dtype=np.int32)])
    return rp, lci, lv


# ------------------------------------------------------------------------------------------
# Device side (one rank's GPU)
# ------------------------------------------------------------------------------------------
def rank_operator(ctx, problem, sh: Shard, form: str = "csr"):
    """The rank's operator on its extended block [halo_lo | own | halo_hi] on the GPU. CSR: the
    extended CSR matrix (halo rows empty). Stencil (slabs of whole z-planes): the same stencil on the
    sub-grid of the extended planes, with the diagonal of those planes; its halo rows are computed
    with the wrong (Dirichlet) neighbours and discarded by the next exchange."""
    from . import runtime as R
    if form == "csr":
        rp, ci, v = problem.csr()
        return R.CsrOperator(ctx, *extended_csr(rp, ci, v, sh))
    plane = problem.nx * problem.ny
    e0, e1 = sh.r0 - sh.lo, sh.r1 + sh.hi
    if e0 % plane or e1 % plane:
        raise ValueError("stencil shards must be whole z-planes")
    dims = (problem.nx, problem.ny, (e1 - e0) // plane) if len(problem.dims) == 3 else (problem.nx, (e1 - e0) // problem.nx)
    kind = {5: 5, 7: 7, 27: 27}[problem.kind]
    return R.StencilOperator(ctx, kind, dims, problem.diag[e0:e1], problem.offdiag, problem.flux,
                             complex_=problem.complex_)


def extended_rows(x_global, sh: Shard):
    """The rank's extended block (rows [r0 - lo, r1 + hi)) of a global row-major block, as a copy."""
    return x_global[sh.r0 - sh.lo:sh.r1 + sh.hi].clone()


def filter_steps(ctx, op_ext, sh: Shard, x_ext, s: int, degree: int, gamma1: float, gamma2: float,
                 precision: str = "fp64"):
    """The rank's side of a sharded filter, one degree step at a time: a generator that runs
    rc_filter_step_rm over the whole extended block and then yields the block x_k whose halo rows
    must be refilled before the next step; after the last step it returns x_m/(m+1) in FP64 (c128)
    as StopIteration.value, converted and scaled as the library's filter does at its end (the
    scale multiplies in double). Ranks advance their generators in lockstep with an exchange
    between yields (sharded_filter does that over torch.distributed)."""
    import torch

    from . import runtime as R
    a, b = gamma2 * gamma1, gamma2
    if degree < 1:
        return x_ext.to(torch.complex128 if x_ext.is_complex() else torch.float64)
    A = x_ext
    B = torch.empty_like(x_ext)
    ld = x_ext.shape[1]
    for k in range(1, degree + 1):
        xk1 = B if (k - 1) % 2 else A   # x_{k-1}
        y = B if k % 2 else A           # x_k over x_{k-2}
        torch.cuda.current_stream().synchronize()  # halo copies of the exchange are on torch's stream
        if k == 1:
            R.filter_step_rm(ctx, op_ext, xk1, None, y, s, a, b, 0.0, precision, ld=ld)
        else:
            R.filter_step_rm(ctx, op_ext, xk1, y, y, s, a, b, -1.0, precision, ld=ld)
        ctx.synchronize()
        yield y
    xm = B if degree % 2 else A
    wide = torch.complex128 if xm.is_complex() else torch.float64
    return xm.to(wide).mul_(1.0 / (degree + 1))


def sharded_filter(ctx, op_ext, sh: Shard, x_ext, s: int, degree: int, gamma1: float, gamma2: float,
                   precision: str = "fp64", group=None):
    """X <- P_m(A')X on the rank's extended row-major block x_ext (ext_rows x ld, storage precision of
    `precision`, halo rows filled), with the recurrence of LanczosCpolyOperatorLMCuda::apply
    (LanczosCpolyOperatorLMCuda.h:194-265): x_1 = a A x_0 + b x_0, x_k = a A x_{k-1} + b x_{k-1} - x_{k-2},
    a = gamma2*gamma1, b = gamma2, result x_m/(m+1). One rc_filter_step_rm per degree over the whole
    extended block, exchange_halo (torch.distributed: NCCL between GPUs) between steps. Every rank
    calls it with the same degree and coefficients. Returns x_m/(m+1) on the extended block in FP64
    (c128); its own rows are the rank's rows of the filtered block."""
    gen = filter_steps(ctx, op_ext, sh, x_ext, s, degree, gamma1, gamma2, precision)
    while True:
        try:
            blk = next(gen)
        except StopIteration as e:
            return e.value
        exchange_halo(blk, sh, group)
