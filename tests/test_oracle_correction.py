"""The correction form of the Chebyshev filter (the MIXED-precision refinement), on the CPU oracle.

x_k = c_k(lambda) v + a e_k rewrites the reference's three-term filter (LanczosCpolyOperatorLM.h:192-304)
on Ritz pairs; e_k carries the residual block R = A V - V diag(lambda) as a source term. In exact
storage the two forms agree to rounding. With R and e_k stored in bfloat16 the filtered block is off
by about 2^-9 times the residual, so its error shrinks as the Ritz pairs converge, while a filter whose
x_k are stored in bfloat16 keeps an error of about 2^-9 at every residual. These are the properties
the GPU solver's bfloat16 correction step relies on."""
import numpy as np
import pytest
import torch

from oracle import rc_oracle as O
from rayleighchebyshevgpgpu_b200 import problems


def _setup(s=12, m=12):
    P = problems.small_laplacian((30, 30), seed=3, vmax=3.0, k=8)
    A = O.csr_matrix(*P.csr())
    w, U = np.linalg.eigh(A.toarray())
    lam_s, lam_max = w[s], w[-1]
    # the recurrence maps [lam_s, lam_max] onto [-2, 2]: a lam + b = 2 at lam_s, -2 at lam_max
    a = -4.0 / (lam_max - lam_s)
    b = 2.0 - a * lam_s
    return A, U[:, :s], b, a / b, m


def _ritz(A, V):
    H = V.T @ (A @ V)
    lam, Q = np.linalg.eigh(0.5 * (H + H.T))
    return V @ Q, lam


def test_round_bf16_is_round_to_nearest_even():
    one = 1.0
    assert O.round_bf16([one])[0] == one
    assert O.round_bf16([one + 2.0 ** -8])[0] == one                       # tie -> even mantissa (0)
    assert O.round_bf16([one + 3 * 2.0 ** -8])[0] == one + 2.0 ** -6        # tie -> even mantissa (2)
    x = np.random.default_rng(1).standard_normal(4096) * np.exp(np.random.default_rng(2).uniform(-30, 30, 4096))
    ref = torch.from_numpy(x.astype(np.float32)).to(torch.bfloat16).to(torch.float64).numpy()
    np.testing.assert_array_equal(O.round_bf16(x), ref)


@pytest.mark.parametrize("m", [1, 2, 3, 12])
def test_correction_form_equals_filter_in_exact_storage(m):
    A, U, g2, g1, _ = _setup(m=m)
    rng = np.random.default_rng(0)
    V, _ = np.linalg.qr(U + 1e-2 * rng.standard_normal(U.shape))
    Y, lam = _ritz(A, V)
    F = O.filter_block(A, Y, m, g1, g2)
    Fc = O.correction_filter(A, Y, lam, m, g1, g2)
    assert np.linalg.norm(Fc - F) <= 1e-13 * np.linalg.norm(F)


def test_bfloat16_correction_error_scales_with_the_residual():
    A, U, g2, g1, m = _setup()
    rng = np.random.default_rng(0)
    N = rng.standard_normal(U.shape)
    rows = []
    for d in (1e-4, 1e-6, 1e-8):
        V, _ = np.linalg.qr(U + d * N)
        Y, lam = _ritz(A, V)
        rn = np.linalg.norm(A @ Y - Y * lam) / np.linalg.norm(Y)
        F = O.filter_block(A, Y, m, g1, g2)
        nf = np.linalg.norm(F)
        err_corr = np.linalg.norm(O.correction_filter(A, Y, lam, m, g1, g2, store=O.round_bf16) - F) / nf
        err_plain = np.linalg.norm(O.filter_block_stored(A, Y, m, g1, g2, O.round_bf16) - F) / nf
        rows.append((rn, err_corr, err_plain))
    for rn, err_corr, err_plain in rows:
        assert err_corr <= 5e-3 * rn, rows          # a few units of 2^-9 times the residual
        assert err_plain >= 1e-3, rows              # the plain bfloat16 filter stays at ~2^-9
    # four orders of magnitude of residual give four orders of magnitude of error
    assert rows[-1][1] <= 1e-3 * rows[0][1], rows
