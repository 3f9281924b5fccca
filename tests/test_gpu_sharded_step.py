"""The device side of the row-sharded filter on one GPU: each rank's degree steps run through
rc_filter_step_rm on its extended block (own rows plus halo rows), and the halo rows are refilled
between steps from the neighbouring ranks' own rows. The ranks are emulated one after another on
one GPU (every rank's step k, then every rank's exchange), so nothing waits on another process.

After m steps every rank's own rows must equal, bit for bit, the unsharded filter: the same step
entry point over the whole operator, and the library's column-major rc_filter (which adds the
layout changes at both ends). 2- and 3-way splits of whole z-planes; CSR (rank operator = the
extended CSR matrix of sharding.extended_csr) and stencils (the stencil on the sub-grid of the
rank's planes plus halo planes); FP64 and FP32 storage. The multi-process exchange over
torch.distributed is covered on gloo ranks (tests/test_sharding_gloo.py)."""
import numpy as np
import pytest

from rayleighchebyshevgpgpu_b200 import problems
from rayleighchebyshevgpgpu_b200 import runtime as R
from rayleighchebyshevgpgpu_b200 import sharding as S

pytestmark = pytest.mark.gpu

DIMS = (14, 11, 12)
S_COLS = 24
DEGREE = 9
G1, G2 = -0.21, 1.7


def _problem(kind):
    n = int(np.prod(DIMS))
    diag = (6.0 if kind == 7 else 1.0) + np.random.default_rng(kind).uniform(0, 2.0, n)
    return problems.Problem(f"shard{kind}", DIMS, kind, diag, -1.0 / 26.0 if kind == 27 else -1.0)


def _rows(x_global, precision):
    """Row-major device block (n x ld) in the storage precision, from a column-major host block."""
    import torch
    ld = R.rm_leading_dim(False, precision, S_COLS)
    dt = torch.float64 if precision == "fp64" else torch.float32
    X = torch.zeros((x_global.shape[1], ld), dtype=dt, device="cuda")
    X[:, :S_COLS] = torch.from_numpy(x_global.T.copy()).to(dt)
    return X


def _exchange_all(blocks, plan):
    """Refill every rank's halo rows from its neighbours' own rows (in-process exchange)."""
    for sh, blk in zip(plan, blocks):
        if sh.lo:
            nb, nsh = blocks[sh.rank - 1], plan[sh.rank - 1]
            blk[:sh.lo] = nb[nsh.lo + nsh.rows - sh.lo:nsh.lo + nsh.rows]
        if sh.hi:
            nb, nsh = blocks[sh.rank + 1], plan[sh.rank + 1]
            blk[sh.lo + sh.rows:] = nb[nsh.lo:nsh.lo + sh.hi]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("form,kind", [("csr", 7), ("stencil", 7), ("stencil", 27)])
@pytest.mark.parametrize("world", [2, 3])
def test_sharded_steps_equal_unsharded_bitwise(ctx, world, form, kind, precision):
    import torch
    P = _problem(kind)
    rp, ci, v = P.csr()
    x0 = np.random.default_rng(5).standard_normal((S_COLS, P.n))  # column-major n x s, as rows
    plan = S.shard_plan(rp, ci, S.partition_rows(P.n, world, quantum=P.nx * P.ny))
    # unsharded: the same step entry point over the whole operator
    op = R.operator_from_problem(ctx, P, form)
    Xg = _rows(x0, precision)
    want = None
    gen = S.filter_steps(ctx, op, S.Shard(0, 1, 0, P.n, 0, 0, 0, 0), Xg, S_COLS, DEGREE, G1, G2, precision)
    try:
        while True:
            next(gen)
    except StopIteration as e:
        want = e.value
    # the library's own column-major filter
    Xc = torch.from_numpy(x0.copy()).cuda()
    torch.cuda.synchronize()  # the library works on its own stream
    R.filter_block(ctx, op, Xc, S_COLS, DEGREE, G1, G2, precision=precision)
    ctx.synchronize()
    assert torch.equal(want[:, :S_COLS].to(torch.float64), Xc.T)
    # sharded, ranks in lockstep with an in-process exchange
    full = _rows(x0, precision)
    ops = [S.rank_operator(ctx, P, sh, form) for sh in plan]
    gens = [S.filter_steps(ctx, o, sh, S.extended_rows(full, sh), S_COLS, DEGREE, G1, G2, precision)
            for o, sh in zip(ops, plan)]
    results = [None] * world
    for _ in range(DEGREE + 1):
        blocks = []
        for r, g in enumerate(gens):
            try:
                blocks.append(next(g))
            except StopIteration as e:
                results[r] = e.value
        if blocks:
            _exchange_all(blocks, plan)
    for sh, res in zip(plan, results):
        own = res[sh.lo:sh.lo + sh.rows]
        assert torch.equal(own, want[sh.r0:sh.r1]), (sh.rank, (own - want[sh.r0:sh.r1]).abs().max().item())
    for o in ops:
        o.close()
    op.close()


def test_step_rejects_bad_leading_dimension(ctx):
    import torch
    P = _problem(7)
    op = R.operator_from_problem(ctx, P, "csr")
    x = torch.zeros((P.n, 6), dtype=torch.float64, device="cuda")  # 6 doubles: not a multiple of 32 bytes
    y = torch.zeros_like(x)
    with pytest.raises(R.capi.RCError):
        R.filter_step_rm(ctx, op, x, None, y, 5, 1.0, 0.0, ld=6)
    op.close()
