"""Kernel-level parity of the correction filter (the MIXED refinement step) on the GPU, through the C
ABI, against the oracle.

rc_filter_correction runs the solver's correction steps on a caller's Ritz pairs: the residual block
R = A V - V diag(lam) (rc_resid.cu, bfloat16), the coefficient tables, the degree steps
(rm_step_src_kernel: bfloat16 storage, FP32 arithmetic) and the FP64 combination. The oracle's
three-term filter (oracle.filter_block, the restatement of LanczosCpolyOperatorLM.h:192-304) and its
correction form with emulated bfloat16 storage (oracle.correction_filter) are the references.

The bound: R and e_k are stored with an 8-bit mantissa, so the filtered block is off by a few units
of 2^-9 times the relative residual rn of the Ritz pairs (tests/test_oracle_correction.py shows the
same bound for the oracle's own bfloat16 form). A wrong coefficient row, a slice offset error or an
off-by-one in the m - 1 steps gives an error of order rn itself, a hundred times the bound.
rc_filter_correction_batch runs the batched kernel (batch_corr_step_kernel); its blocks must equal
the single-block kernel's bit for bit."""
import numpy as np
import pytest

from oracle import rc_oracle as O
from rayleighchebyshevgpgpu_b200 import problems
from rayleighchebyshevgpgpu_b200 import runtime as R

pytestmark = pytest.mark.gpu

BOUND = 5e-3  # x the relative residual of the Ritz pairs, relative to ||filtered block||

_CASES = {
    "csr7": (7, (14, 13, 12)),
    "st5": (5, (46, 41)),
    "st7": (7, (14, 13, 12)),
    "st27": (27, (12, 11, 10)),
}
# complex Hermitian tight-binding operators with Peierls phases on the y-bonds (flux 1/17 and 0.11)
_CCASES = {
    "ccsr7": ((13, 12, 11), 1.0 / 17.0),
    "cst7": ((13, 12, 11), 1.0 / 17.0),
    "cst5": ((43, 39), 0.11),
}
_cache = {}


def _problem(name):
    if name not in _cache:
        if name in _CCASES:
            dims, flux = _CCASES[name]
            Q = problems.small_laplacian(dims, seed=len(dims) + 40, complex_=True, flux=flux)
        else:
            kind, dims = _CASES[name]
            n = int(np.prod(dims))
            rng = np.random.default_rng(kind * 7 + len(dims))
            d0 = {5: 4.0, 7: 6.0, 27: 1.0}[kind]
            diag = d0 + rng.uniform(0.0, 3.0 if kind != 27 else 2.0, n)
            Q = problems.Problem(name, dims, kind, diag, -1.0 / 26.0 if kind == 27 else -1.0)
        A = O.csr_matrix(*Q.csr())
        w, U = np.linalg.eigh(A.toarray())
        _cache[name] = (Q, A, w, U)
    return _cache[name]


def _ritz_pairs(A, U, s, d, seed):
    """Ritz pairs of a perturbed invariant subspace: residual about d (complex U: complex noise)."""
    rng = np.random.default_rng(seed)
    noise = rng.standard_normal((U.shape[0], s))
    if np.iscomplexobj(U):
        noise = noise + 1j * rng.standard_normal((U.shape[0], s))
    V, _ = np.linalg.qr(U[:, :s] + d * noise)
    H = V.conj().T @ (A @ V)
    lam, Qs = np.linalg.eigh(0.5 * (H + H.conj().T))
    Y = V @ Qs
    rn = np.linalg.norm(A @ Y - Y * lam) / np.linalg.norm(Y)
    return Y, lam, rn


def _coefficients(w, s, m):
    """(gamma1, gamma2) mapping [w[s], w[-1]] onto [-2, 2] for the recurrence a lam + b."""
    a = -4.0 / (w[-1] - w[s])
    b = 2.0 - a * w[s]
    return a / b, b


def _op(ctx, Q, name):
    return R.operator_from_problem(ctx, Q, "csr" if "csr" in name else "stencil")


def _gpu(ctx, op, Y, s, lam, m, g1, g2):
    import torch
    Vd = torch.from_numpy(np.ascontiguousarray(Y.T)).cuda()  # column-major n x s
    R.filter_correction(ctx, op, Vd, s, lam, m, g1, g2)
    return Vd.cpu().numpy().T


def _check(A, Y, lam, rn, m, g1, g2, got):
    F = O.filter_block(A, Y, m, g1, g2)
    Fb = O.correction_filter(A, Y, lam, m, g1, g2, store=O.round_bf16)
    nf = np.linalg.norm(F)
    err_exact = np.linalg.norm(got - F) / nf
    err_bf16 = np.linalg.norm(got - Fb) / nf
    assert err_exact <= BOUND * rn, (err_exact, rn)
    assert err_bf16 <= BOUND * rn, (err_bf16, rn)
    return err_exact


@pytest.mark.parametrize("name", list(_CASES))
@pytest.mark.parametrize("s", [5, 8, 24, 48, 96])
def test_correction_filter_matches_oracle(ctx, name, s):
    Q, A, w, U = _problem(name)
    m = 9
    Y, lam, rn = _ritz_pairs(A, U, s, 1e-5, seed=s)
    g1, g2 = _coefficients(w, s, m)
    op = _op(ctx, Q, name)
    got = _gpu(ctx, op, Y, s, lam, m, g1, g2)
    _check(A, Y, lam, rn, m, g1, g2, got)
    op.close()


@pytest.mark.parametrize("name", list(_CCASES))
@pytest.mark.parametrize("s", [4, 24, 96, 192])
def test_complex_correction_filter_matches_oracle(ctx, name, s):
    """Complex Hermitian operators: complex bfloat16 blocks (real and imaginary part each a bfloat16),
    c64 arithmetic, real Ritz values and coefficients, up to the 192 columns of the 96^3 complex
    tight-binding workload."""
    Q, A, w, U = _problem(name)
    m = 9
    Y, lam, rn = _ritz_pairs(A, U, s, 1e-5, seed=s + 3)
    g1, g2 = _coefficients(w, s, m)
    op = _op(ctx, Q, name)
    got = _gpu(ctx, op, Y, s, lam, m, g1, g2)
    _check(A, Y, lam, rn, m, g1, g2, got)
    op.close()


@pytest.mark.parametrize("name", ["csr7", "st7", "st27"])
@pytest.mark.parametrize("s", [130, 256])
def test_wide_correction_filter_matches_oracle(ctx, name, s):
    """Real blocks wider than 96 columns: the row-major FP64 copy of V comes from a layout change
    and the residual block kernel takes one 16-byte slice per thread or two."""
    Q, A, w, U = _problem(name)
    m = 7
    Y, lam, rn = _ritz_pairs(A, U, s, 1e-5, seed=s)
    g1, g2 = _coefficients(w, s, m)
    op = _op(ctx, Q, name)
    got = _gpu(ctx, op, Y, s, lam, m, g1, g2)
    _check(A, Y, lam, rn, m, g1, g2, got)
    op.close()


@pytest.mark.parametrize("m", [1, 2, 3, 41])
def test_correction_filter_degrees(ctx, m):
    Q, A, w, U = _problem("csr7")
    s = 24
    Y, lam, rn = _ritz_pairs(A, U, s, 1e-4, seed=m)
    g1, g2 = _coefficients(w, s, m)
    op = _op(ctx, Q, "csr7")
    got = _gpu(ctx, op, Y, s, lam, m, g1, g2)
    _check(A, Y, lam, rn, m, g1, g2, got)
    op.close()


def test_correction_error_shrinks_with_the_residual(ctx):
    """The defining property: the error follows the residual down (1e-3 -> 1e-7), where a filter
    stored in bfloat16 would stay at about 2^-9."""
    Q, A, w, U = _problem("st7")
    s, m = 24, 12
    g1, g2 = _coefficients(w, s, m)
    op = _op(ctx, Q, "st7")
    errs = []
    for d in (1e-3, 1e-5, 1e-7):
        Y, lam, rn = _ritz_pairs(A, U, s, d, seed=11)
        errs.append(_check(A, Y, lam, rn, m, g1, g2, _gpu(ctx, op, Y, s, lam, m, g1, g2)))
    assert errs[-1] <= 1e-2 * errs[0], errs
    op.close()


def test_batched_correction_equals_single_block_bitwise(ctx):
    """Two different jobs (CSR s = 24, degree 9; 7-point stencil s = 48, degree 13) in one batched
    launch per step, plus a 27-point job and a complex job that run on the single-block kernels in
    the same call: every block equals its rc_filter_correction result bit for bit and matches the
    oracle."""
    import torch
    jobs, singles, refs = [], [], []
    for name, s, m, seed in (("csr7", 24, 9, 1), ("st7", 48, 13, 2), ("st27", 16, 7, 3), ("cst7", 20, 8, 4)):
        Q, A, w, U = _problem(name)
        Y, lam, rn = _ritz_pairs(A, U, s, 1e-5, seed=seed)
        g1, g2 = _coefficients(w, s, m)
        op = _op(ctx, Q, name)
        singles.append(_gpu(ctx, op, Y, s, lam, m, g1, g2))
        Vd = torch.from_numpy(np.ascontiguousarray(Y.T)).cuda()
        jobs.append((op, Vd, s, lam, m, g1, g2))
        refs.append((A, Y, lam, rn, m, g1, g2))
    batched = R.filter_correction_batch(ctx, jobs)
    assert batched == 2
    for (op, Vd, *_), single, ref in zip(jobs, singles, refs):
        got = Vd.cpu().numpy().T
        assert np.array_equal(got, single)
        _check(*ref, got)
        op.close()


def test_correction_filter_rejects_unsupported(ctx):
    """Blocks wider than 256 columns are refused (RC_ERR_UNSUPPORTED), before any work."""
    import torch
    Q = problems.small_laplacian((8, 8, 8), seed=1, complex_=True, flux=0.1)
    op = R.operator_from_problem(ctx, Q, "csr")
    s = 257
    Vd = torch.zeros((s, Q.n), dtype=torch.complex128, device="cuda")
    with pytest.raises(R.capi.RCError) as e:
        R.filter_correction(ctx, op, Vd, s, np.zeros(s), 3, 0.1, 1.0)
    assert e.value.status == 8  # RC_ERR_UNSUPPORTED
    op.close()


@pytest.mark.parametrize("name", ["csr7", "st7", "st5", "cst7", "ccsr7"])
@pytest.mark.parametrize("m", [3, 8, 13])
def test_two_step_kernel_equals_one_step_launches_bitwise(name, m):
    """The correction filter's degree steps two per launch (rm_corr2_kernel: phase A of a block, phase B
    of a block behind it, ordered by per-group completion counters) give the same bits as one launch
    per step (RCB200_CORR_PAIR=0): the same arithmetic per row, e_k read back before DRAM. Odd and even
    step counts (the last step of an even count runs alone)."""
    import os
    import torch
    Q, A, w, U = _problem(name)
    s = 24 if name.startswith("c") else 40
    Y, lam, rn = _ritz_pairs(A, U, s, 1e-5, seed=m)
    g1, g2 = _coefficients(w, s, m)
    out = []
    for flag in ("1", "0"):
        old = os.environ.get("RCB200_CORR_PAIR")
        os.environ["RCB200_CORR_PAIR"] = flag
        try:
            c = R.Context(0)
        finally:
            if old is None:
                os.environ.pop("RCB200_CORR_PAIR", None)
            else:
                os.environ["RCB200_CORR_PAIR"] = old
        op = _op(c, Q, name)
        got = _gpu(c, op, Y, s, lam, m, g1, g2)
        assert (c.counter("pair_launches") > 0) == (flag == "1")
        out.append(got)
        op.close()
        c.close()
    assert np.array_equal(out[0], out[1])
    _check(A, Y, lam, rn, m, g1, g2, out[0])


@pytest.mark.parametrize("dims", [(12, 11, 10), (33, 7, 5)])
@pytest.mark.parametrize("s", [8, 24, 48, 80])
def test_27_point_warp_rows_equal_thread_runs_bitwise(dims, s):
    """The 27-point correction step with a warp's lanes on consecutive rows (cross-section sums of
    neighbouring rows passed by shuffles) gives the same bits as the per-thread runs of 16 rows
    (RCB200_ROWS27W=0): the same sums in the same order. Rows of 1, 3, 6 and 10 bfloat16 slices (32,
    10, 5 and 3 rows per warp step), on grids whose x-lines and row counts do not divide the steps."""
    import os
    n = int(np.prod(dims))
    rng = np.random.default_rng(s + n)
    Q = problems.Problem("st27w", dims, 27, 1.0 + rng.uniform(0.0, 2.0, n), -1.0 / 26.0)
    A = O.csr_matrix(*Q.csr())
    X = rng.standard_normal((n, s))
    Y, _ = np.linalg.qr(X)
    H = Y.T @ (A @ Y)
    lam, Qs = np.linalg.eigh(0.5 * (H + H.T))
    Y = Y @ Qs
    out = []
    for flag in ("1", "0"):
        old = os.environ.get("RCB200_ROWS27W")
        os.environ["RCB200_ROWS27W"] = flag
        try:
            c = R.Context(0)
        finally:
            if old is None:
                os.environ.pop("RCB200_ROWS27W", None)
            else:
                os.environ["RCB200_ROWS27W"] = old
        op = R.operator_from_problem(c, Q, "stencil")
        out.append(_gpu(c, op, Y, s, lam, 9, -0.3, 1.1))
        op.close()
        c.close()
    assert np.all(np.isfinite(out[0]))
    assert np.array_equal(out[0], out[1])
