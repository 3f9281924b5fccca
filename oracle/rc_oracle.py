"""ORACLE -- CPU restatement of the reference's Rayleigh-Chebyshev path, for tests only.

Test infrastructure: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
import this module, and only as the checker. The product path never calls it.

Each function restates the reference routine it cites (paths relative to the reference project):
  pm, pm_prime, pm_prime_first_root, inverse_pm, xstar, upper_xstar, star_degree_and_bound
      LanczosCpoly.h:234-270, :400-415, :371-398, :416-473, :285-305, :498-555
  filter_block   LanczosCpolyOperatorLM.h:192-304 (same recurrence as LanczosCpolyOperatorLMCuda.h:194-265)
  correction_filter  no reference counterpart: the same filter written on Ritz pairs as
                 x_k = c_k(lambda) v + a e_k (the MIXED-precision correction form), with the storage
                 rounding of R and e_k as a parameter (round_bf16 emulates bfloat16 storage)
  lanczos_bounds LanczosMaxMinFinder.h:248-544 (tridiagonal extremes by LAPACK dstebz there,
                 by scipy's eigvalsh_tridiagonal here)
  solve          RayleighChebyshevLM.h:712-1776 (getMinEigenSystem and its base routine), with the
                 projected eigenproblem by LAPACK (numpy.linalg.eigh) as in the LAPACK build
                 (RayleighChebyshevLM.h:490-518)

Parity is pinned by tests/test_oracle.py: against the reference compiled from its own sources
(oracle/_ref, built by oracle/Makefile) and against dense LAPACK eigenvalues / analytic spectra.
"""
from __future__ import annotations

import math

import numpy as np
import scipy.linalg as sla
import scipy.sparse as sp

SMALL_TOL = 1.0e-11          # RAYLEIGH_CHEBYSHEV_SMALL_TOL_ (RayleighChebyshevLMCuda.h:210)
LANCZOS_SMALL_TOL = 1.0e-10  # LANCZOS_SMALL_TOL_ (LanczosMaxMinFinder.h:76)
PI_TRUNC = 3.14159265359      # the truncated pi of LanczosCpoly.h:431,438


# ------------------------------------------------------------------------------------------
# LanczosCpoly.h
# ------------------------------------------------------------------------------------------
def pm(m: int, x: float) -> float:
    """P_m(x) = b_m/(m+1), b_k = (2-4x) b_{k-1} - b_{k-2} (LanczosCpoly.h:234-270)."""
    if m == 0:
        return 1.0
    if m == 1:
        return 1.0 - 2.0 * x
    c = 2.0 - 4.0 * x
    b0, b1 = 1.0, c
    for _ in range(2, m + 1):
        b0, b1 = b1, c * b1 - b0
    return b1 / (m + 1)


def pm_prime(m: int, x: float) -> float:
    """dP_m/dx in closed form through theta with sin^2(theta/2) = x (LanczosCpoly.h:400-415)."""
    mp = m + 1.0
    h = math.asin(math.sqrt(x))            # theta/2
    s2 = math.sin(2.0 * h)                 # sin(theta)
    dtheta_dx = 1.0 / (math.sqrt(x) * math.sqrt(1.0 - x))
    dp_dtheta = (math.cos(2.0 * mp * h) / s2 - math.sin(2.0 * mp * h) * math.cos(2.0 * h) / (mp * s2 * s2))
    return dp_dtheta * dtheta_dx


def _secant(f, xa, xb, tol=1e-12, maxit=200):
    fa, fb = f(xa), f(xb)
    it = 0
    while abs(xa - xb) > tol and it < maxit:
        d = (fb - fa) / (xb - xa)
        xc = xb - fb / d
        xa, fa = xb, fb
        xb, fb = xc, f(xc)
        it += 1
    return xb


def pm_prime_first_root(m: int) -> float:
    """Secant from the sinc-extremum guess 4.49^2/(4(m+1)^2) (LanczosCpoly.h:371-398)."""
    xa = 4.49 * 4.49 / (4.0 * (m + 1) * (m + 1))
    xb = 4.49 * 4.49 / (4.0 * m * (m + 1))
    return _secant(lambda x: pm_prime(m, x), xa, xb)


def inverse_pm(m: int, y: float) -> float:
    """x <= first root with P_m(x) = y; log-transformed for y > 5 (LanczosCpoly.h:416-473)."""
    s1 = math.sin(0.5 * (PI_TRUNC / (m + 1)))
    if y < 0.0:
        return s1 * s1
    if y <= 5.0:
        xa, fa = 0.0, 1.0
        xb, fb = s1 * s1, 0.0
        it = 0
        while abs(xa - xb) > 1e-12 and it < 200:
            d = (fb - fa) / (xb - xa)
            xc = xb - (pm(m, xb) - y) / d
            xa, fa = xb, fb
            xb = xc
            fb = pm(m, xb)
            it += 1
        return xb
    xa, fa = 0.0, 0.0
    xb = -4.0 / ((m + 1.0) * (m + 1.0))
    fb = math.log(pm(m, xb))
    it = 0
    while abs(xa - xb) > 1e-12 and it < 200:
        d = (fb - fa) / (xb - xa)
        xc = xb - (math.log(pm(m, xb)) - math.log(y)) / d
        xa, fa = xb, fb
        xb = xc
        fb = math.log(pm(m, xb))
        it += 1
    return xb


def xstar(m: int) -> float:
    """LanczosCpoly::getXStar (LanczosCpoly.h:285-293)."""
    if m == 0:
        return 1.0
    if m == 1:
        return 0.3
    xp = pm_prime_first_root(m)
    return inverse_pm(m, -pm(m, xp))


def upper_xstar(m: int) -> float:
    """LanczosCpoly::getUpperXStar (LanczosCpoly.h:295-305, :363-369)."""
    if m == 0:
        return 1.0
    if m == 1:
        return 0.6
    if m == 2:
        return (1.0 - xstar(2) + 0.6) / 2.0
    return (math.cos((2.0 / (m + 1.0)) * 3.1415926535897932384) + 1.0) * 0.5


_RATIO_CACHE: dict[int, float] = {}


def _ratio(m: int) -> float:
    if m not in _RATIO_CACHE:
        _RATIO_CACHE[m] = xstar(m) / upper_xstar(m)
    return _RATIO_CACHE[m]


def star_degree_and_bound(shift: float, lambda_bound: float, lambda_star: float, deg_max: int):
    """LanczosCpoly::getStarDegreeAndSpectralRadius (LanczosCpoly.h:498-555)."""
    lss = lambda_star + shift
    r = _ratio(1)
    if r * (lambda_bound + shift) < lss:
        return 1, lss / r - shift
    mb = 2
    while mb < deg_max:
        if _ratio(mb) * (lambda_bound + shift) < lss:
            break
        mb += 1
    if mb >= deg_max:
        return deg_max, lambda_bound
    return mb, lss / _ratio(mb) - shift


def gammas(m: int, lambda_max: float, shift: float):
    """gamma1, gamma2 of LanczosCpolyOperatorLM(Cuda)::apply (LanczosCpolyOperatorLM.h:201-206)."""
    ux = upper_xstar(m)
    rho = lambda_max / ux + shift / ux
    return -2.0 / (rho - 2.0 * shift), 2.0 - 4.0 * shift / rho


# ------------------------------------------------------------------------------------------
# LanczosCpolyOperatorLM.h
# ------------------------------------------------------------------------------------------
def filter_block(A, X: np.ndarray, m: int, g1: float, g2: float, reps: int = 1) -> np.ndarray:
    """Apply P_m(A') to the columns of X (n x s): x1 = g2(g1 A x0 + x0),
    x_k = g2(g1 A x_{k-1} + x_{k-1}) - x_{k-2}, result x_m/(m+1) (LanczosCpolyOperatorLM.h:192-304)."""
    V = np.array(X, copy=True)
    for _ in range(reps):
        vnm2 = V.copy()
        vnm1 = g2 * (g1 * (A @ V) + V)
        for _k in range(2, m + 1):
            vn = g2 * (g1 * (A @ vnm1) + vnm1) - vnm2
            vnm2, vnm1 = vnm1, vn
        V = vnm1 * (1.0 / (m + 1))
    return V


def round_bf16(x) -> np.ndarray:
    """Values rounded to bfloat16 (round to nearest, ties to even, via float32), returned as float64:
    the storage rounding of the correction filter's blocks. Complex values round their real and
    imaginary parts separately (complex128 out)."""
    if np.iscomplexobj(x):
        return round_bf16(np.real(x)) + 1j * round_bf16(np.imag(x))
    f = np.ascontiguousarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def correction_filter(A, V: np.ndarray, lam: np.ndarray, m: int, g1: float, g2: float, store=None) -> np.ndarray:
    """filter_block(A, V, m, g1, g2) written on Ritz pairs (v_c, lam_c). With a = g2 g1, b = g2 and the
    scalar recurrence c_0 = 1, c_1 = a lam + b, c_k = (a lam + b) c_{k-1} - c_{k-2}, the filter's
    x_k = (aA + b) x_{k-1} - x_{k-2} is x_k = c_k v + a e_k with
        e_0 = 0, e_1 = R = A V - V diag(lam), e_k = (aA + b) e_{k-1} - e_{k-2} + c_{k-1} R,
    and the result is x_m/(m+1) = (c_m v + a e_m)/(m+1). `store` rounds R and every e_k as stored
    (None: exact); the rest is float64. No reference counterpart (the MIXED-precision refinement)."""
    rnd = store if store is not None else (lambda x: x)
    a, b = g2 * g1, g2
    lam = np.asarray(lam, dtype=np.float64)
    R = rnd(A @ V - V * lam)
    t = a * lam + b
    cm2, cm1 = np.ones_like(lam), t.copy()  # c_0, c_1
    em2, em1 = np.zeros_like(V), R            # e_0, e_1
    for _k in range(2, m + 1):
        ek = rnd(a * (A @ em1) + b * em1 - em2 + cm1 * R)
        cm2, cm1 = cm1, t * cm1 - cm2
        em2, em1 = em1, ek
    return (cm1 * V + a * em1) / (m + 1)


def filter_block_stored(A, X: np.ndarray, m: int, g1: float, g2: float, store) -> np.ndarray:
    """filter_block with every intermediate x_k rounded by `store` (the plain reduced-precision
    filter, for comparison with correction_filter)."""
    V = store(np.array(X, copy=True))
    vnm2 = V
    vnm1 = store(g2 * (g1 * (A @ V) + V))
    for _k in range(2, m + 1):
        vn = store(g2 * (g1 * (A @ vnm1) + vnm1) - vnm2)
        vnm2, vnm1 = vnm1, vn
    return vnm1 * (1.0 / (m + 1))


# ------------------------------------------------------------------------------------------
# LanczosMaxMinFinder.h
# ------------------------------------------------------------------------------------------
def _lz_rel(val, tol):
    return abs(val) if abs(val) * tol > LANCZOS_SMALL_TOL else LANCZOS_SMALL_TOL / tol


def lanczos_bounds(A, v0: np.ndarray, tol: float = 1e-6, which: str = "max", max_iter: int = 10000):
    """LanczosMaxMinFinder::getMinMaxEigenvalues (LanczosMaxMinFinder.h:248-544)."""
    tol = min(tol, 0.01)
    tol = max(tol, LANCZOS_SMALL_TOL)
    v = np.array(v0, dtype=np.result_type(v0, A.dtype), copy=True)
    v /= math.sqrt(abs(np.vdot(v, v)))
    w = v.copy()
    v[:] = 0
    alpha, beta = [], []
    min_diff = max_diff = 1e10
    lmin = lmax = 0.0
    rf_max = rf_min = 9.0
    r_max = r_min = 1.0
    emax_old = emin_old = 0.0
    dmax_a = dmin_a = dmax_b = dmin_b = 0.0
    diff_cmp = rate_cmp = 0
    k = 0
    done = False
    while k < max_iter and not done:
        if k != 0 and abs(beta[k - 1]) > 1e-14:
            wt = w.copy()
            w = v / beta[k - 1]
            v = -beta[k - 1] * wt
        v = v + A @ w
        ak = np.vdot(v, w)  # w.dot(v) = sum w conj(v)
        if abs(ak.imag) > (1.0 + abs(ak.real)) * 1e-12:
            raise ValueError("operator not Hermitian")
        alpha.append(ak.real)
        v = v - ak.real * w
        beta.append(math.sqrt(abs(np.vdot(v, v))))
        k += 1
        if k % 5 == 0:
            ev = sla.eigvalsh_tridiagonal(np.array(alpha), np.array(beta[:k - 1]))
            lmax, lmin = ev[-1], ev[0]
            if diff_cmp == 0:
                emax_old, emin_old = lmax, lmin
                diff_cmp = 1
            else:
                max_diff = abs(lmax - emax_old) / _lz_rel(lmax, tol)
                min_diff = abs(lmin - emin_old) / _lz_rel(lmin, tol)
                if rate_cmp == 0:
                    dmax_a, dmin_a = abs(lmax - emax_old), abs(lmin - emin_old)
                    rate_cmp = 1
                else:
                    if max_diff > 1e-9:
                        dmax_b = abs(lmax - emax_old)
                        r_max = dmax_b / dmax_a
                    else:
                        r_max = 0.95
                    if min_diff > 1e-9:
                        dmin_b = abs(lmin - emin_old)
                        r_min = dmin_b / dmin_a
                    else:
                        r_min = 0.95
                    rf_max = r_max / (1 - r_max) if r_max < 0.9 else 9.0
                    rf_min = r_min / (1 - r_min) if r_min < 0.9 else 9.0
                    dmax_a, dmin_a = dmax_b, dmin_b
                emax_old, emin_old = lmax, lmin
                min_diff *= rf_min
                max_diff *= rf_max
            if which == "both":
                done = min_diff < tol and max_diff < tol
            elif which == "max":
                done = max_diff < tol
            else:
                done = min_diff < tol
    if lmin > lmax:
        lmin, lmax = lmax, lmin
    return lmin, lmax, k


# ------------------------------------------------------------------------------------------
# RayleighChebyshevLM.h -- getMinEigenSystem (single outer pass and multi-pass)
# ------------------------------------------------------------------------------------------
def _rel(val, tol):
    return abs(val) if abs(val) * tol > SMALL_TOL else SMALL_TOL / tol


def _orth(V):
    q, _ = np.linalg.qr(V)
    return q


def solve(A, k: int, tol: float, incr: int, buffer: int, V0: np.ndarray, lz0: np.ndarray,
          stop: str = "RESIDUAL_ONLY", deg_max: int = 200, max_inner: int = 10000, max_min_tol: float = 1e-6,
          verbose: bool = False):
    """Restatement of RayleighChebyshevLM::getMinEigenSystem(eigCount, tol, incr, buffer, ...)
    (RayleighChebyshevLM.h:712-739 -> base routine :817-1776) for small n. V0: n x s start block.
    Returns dict with eigenvalues, eigenvectors (n x found), residuals and counters."""
    n = A.shape[0]
    lmin, lmax, lz_it = lanczos_bounds(A, lz0, max_min_tol, "max")
    if abs(lmax - lmin) > 1e-12:
        lmax += 0.001 * abs(lmax - lmin)
    min_eig, lambda_max, max_eig = lmin, lmax, lmax
    tol = max(tol, SMALL_TOL)
    ss = incr + buffer
    if ss > n:
        if incr < n:
            buffer = n - incr
            ss = n
        else:
            ss = incr = n
            buffer = 0
        k = n
    V = np.array(V0[:, :ss], copy=True)
    old = np.zeros(ss)
    diffs = np.ones(ss)
    olddiffs = np.ones(ss)
    found_vals, found_vecs, found_res = [], [], []
    rng = np.random.default_rng(12345)
    exit_flag = False
    star_degree, star_bound = 0, 0.0
    apply_cum = 0
    inner_total = 0
    degree_steps = 0
    last_found = 0
    while not exit_flag:
        if buffer < ss:
            old[buffer:ss] = old[buffer]  # RayleighChebyshevLM.h:1075-1078
        if apply_cum > 0 and last_found > 0:
            V[:, ss - last_found:] = rng.uniform(-1, 1, (n, last_found))
        E = np.column_stack(found_vecs) if found_vecs else None

        def deflate(X):
            if E is None:
                return X
            for _ in range(2):
                X = X - E @ (E.conj().T @ X)
            return X

        V = _orth(deflate(V))
        lam_star = max_eig
        ratio = 1.0
        it = 0
        deg_save, bound_save = 0, 0.0
        stop_val = tol + 1e10
        hist = []
        max_gap = max_res = max_diff = 0.0
        osc = 0
        while stop_val > tol and it < max_inner:
            shift = -min_eig
            deg_save, bound_save = star_degree, star_bound
            star_degree = 0
            emin = abs(min_eig - lam_star) / _rel(min_eig, tol)
            emax = abs(max_eig - lam_star) / _rel(max_eig, tol)
            if emin < tol and emax < tol:
                star_degree, star_bound = 1, max_eig
            elif (not (max_diff > tol)) and it > 3 and ratio < 0.2:
                star_degree, star_bound = deg_save, bound_save
            if star_degree == 0:
                star_degree, star_bound = star_degree_and_bound(shift, max_eig, lam_star, deg_max)
            if star_degree < deg_save:
                star_degree, star_bound = deg_save, bound_save
            g1, g2 = gammas(star_degree, star_bound, shift)
            V = filter_block(A, V, star_degree, g1, g2)
            degree_steps += star_degree
            V = _orth(deflate(V))
            AV = A @ V
            H = V.conj().T @ AV
            H = 0.5 * (H + H.conj().T)
            lam, Q = np.linalg.eigh(H)
            V = V @ Q
            AV = A @ V
            rcount = incr if len(found_vals) + ss < n else ss
            res = np.linalg.norm(AV[:, :rcount] - V[:, :rcount] * lam[:rcount], axis=0)
            max_res = max([res[j] / _rel(lam[j], tol) for j in range(rcount)] + [0.0])
            hist.append(max_res)
            chk = min(incr, ss)
            olddiffs[:chk] = diffs[:chk]
            max_diff = 0.0
            for i in range(chk):
                d = abs(lam[i] - old[i]) / _rel(old[i], tol)
                diffs[i] = d
                max_diff = max(max_diff, d)
            old[:ss] = lam
            ratio = 0.0
            if max_diff > tol:
                cnt = 0
                for i in range(chk):
                    if abs(olddiffs[i]) > tol / 10:
                        ratio += abs(diffs[i] / olddiffs[i])
                        cnt += 1
                ratio = ratio / cnt if cnt else 1.0
            if stop == "RESIDUAL_ONLY":
                stop_val = max_res
            elif stop == "EIGENVALUE_ONLY":
                stop_val = max_diff
            else:
                stop_val = max_diff if max_res <= math.sqrt(tol) else max_res
            if stop == "RESIDUAL_ONLY" and max_res < math.sqrt(tol) and len(hist) - 1 > 3:
                r = len(hist) - 1
                a = (hist[r - 3] - 2 * hist[r - 2] + hist[r - 1]) / abs(max_res)
                b = (hist[r - 2] - 2 * hist[r - 1] + hist[r]) / abs(max_res)
                if a * b < 0:
                    osc += 1
                    if osc > 5:
                        stop_val = 0.0
            lam_star = lam[ss - 1]
            min_eig = min(min_eig, lam[0])
            it += 1
            if verbose:
                print(f"{it:4d} deg {star_degree:3d} res {max_res:.3e} diff {max_diff:.3e}")
        inner_total += it
        apply_cum += it
        nfound_before = len(found_vals)
        chkc = incr if nfound_before + ss < n else ss
        fc = sum(1 for i in range(chkc) if (lam[i] - lambda_max) / _rel(lambda_max, tol) < tol)
        if fc + nfound_before >= k:
            fc = k - nfound_before
            exit_flag = True
        if fc + nfound_before >= n:
            fc = n - nfound_before
            exit_flag = True
        for i in range(fc):
            found_vals.append(lam[i])
            found_vecs.append(V[:, i].copy())
            found_res.append(res[i] if i < len(res) else 0.0)
        if not exit_flag and fc > 0:
            V = np.column_stack([V[:, fc:], V[:, :fc]])
        last_found = fc
        guard = lam[ss - buffer] if buffer > 0 else lambda_max
        if guard > lambda_max:
            exit_flag = True
        if found_vals:
            min_eig = found_vals[-1]
        star_degree, star_bound = 1, max_eig
        if not exit_flag and len(found_vals) + ss >= n:
            exit_flag = True  # small-n end game not needed by the tests
    return {
        "eigenvalues": np.array(found_vals),
        "eigenvectors": np.column_stack(found_vecs) if found_vecs else np.zeros((n, 0)),
        "residuals": np.array(found_res),
        "inner_iterations": inner_total,
        "degree_steps": degree_steps,
        "lanczos_iterations": lz_it,
        "bounds": (lmin, lmax),
    }


# ------------------------------------------------------------------------------------------
# helpers for the checks
# ------------------------------------------------------------------------------------------
def csr_matrix(rowptr, colind, vals):
    n = len(rowptr) - 1
    return sp.csr_matrix((vals, colind, rowptr), shape=(n, n))


def dense_lowest(A, k: int) -> np.ndarray:
    """Lowest k eigenvalues by dense LAPACK (?syevr/?heevr) -- the small-n oracle."""
    D = A.toarray() if sp.issparse(A) else np.asarray(A)
    return sla.eigh(D, eigvals_only=True, subset_by_index=(0, k - 1), driver="evr")


def laplacian_1d_dirichlet(n: int, k: int) -> np.ndarray:
    """Analytic lowest eigenvalues of tridiag(-1, 2, -1) of size n: 2 - 2cos(j pi/(n+1))."""
    j = np.arange(1, k + 1)
    return 2.0 - 2.0 * np.cos(j * np.pi / (n + 1))


def max_subspace_angle(U: np.ndarray, V: np.ndarray) -> float:
    """Largest principal angle between the column spaces of U and V (columns normalised first)."""
    Un = U / np.linalg.norm(U, axis=0)
    Vn = V / np.linalg.norm(V, axis=0)
    qu, _ = np.linalg.qr(Un)
    qv, _ = np.linalg.qr(Vn)
    s = np.linalg.svd(qu.conj().T @ qv, compute_uv=False)
    return float(np.arccos(np.clip(s.min(), -1.0, 1.0)))
