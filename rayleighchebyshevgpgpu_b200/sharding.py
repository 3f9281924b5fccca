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
The device side of the sharded solve (the degree-step kernel reading the extended block, with the
exchange between steps) is not part of this build: every run here has one GPU.
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
