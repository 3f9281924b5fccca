"""Python host layer over the C ABI: context, operators and the whole-solve call.

Device blocks passed to the kernel-level calls are raw device pointers (for example
``torch.Tensor.data_ptr()`` of a CUDA tensor); whole solves can also take host numpy arrays
(``host=True``), in which case the library performs the host<->device copies.
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, Optional

import numpy as np

from . import _capi as capi
from ._capi import check, lib

_STOP = {"DEFAULT": capi.RC_STOP_DEFAULT, "COMBINATION": capi.RC_STOP_COMBINATION,
         "EIGENVALUE_ONLY": capi.RC_STOP_EIGENVALUE_ONLY, "RESIDUAL_ONLY": capi.RC_STOP_RESIDUAL_ONLY}
_PREC = {"fp64": capi.RC_PREC_FP64, "mixed": capi.RC_PREC_MIXED}


def _ptr(a) -> int:
    """Address of a numpy array or torch tensor (or an int address)."""
    if a is None:
        return 0
    if isinstance(a, int):
        return a
    if hasattr(a, "data_ptr"):
        return int(a.data_ptr())
    if isinstance(a, np.ndarray):
        return int(a.ctypes.data)
    raise TypeError(f"cannot take the address of {type(a)}")


class Context:
    """A device, a stream and the workspace arena (rc_ctx)."""

    def __init__(self, device: int = 0):
        self.h = C.c_void_p()
        check(lib().rc_ctx_create(device, C.byref(self.h)), None, "rc_ctx_create")
        self.device = device

    def close(self):
        if self.h:
            lib().rc_ctx_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def synchronize(self):
        check(lib().rc_ctx_synchronize(self.h), self.h, "synchronize")

    def set_stream(self, stream_ptr: int | None):
        check(lib().rc_ctx_set_stream(self.h, C.c_void_p(stream_ptr or 0)), self.h, "set_stream")

    def launches(self, reset: bool = False) -> int:
        v = C.c_int64()
        check(lib().rc_ctx_launch_count(self.h, C.byref(v), 1 if reset else 0), self.h)
        return v.value

    def counter(self, name: str) -> int:
        v = C.c_int64()
        check(lib().rc_ctx_counter(self.h, name.encode(), C.byref(v)), self.h, "rc_ctx_counter")
        return v.value

    def device_bytes(self) -> int:
        v = C.c_int64()
        check(lib().rc_ctx_device_bytes(self.h, C.byref(v)), self.h)
        return v.value

    def last_error(self) -> str:
        raw = lib().rc_ctx_last_error(self.h)
        return raw.decode() if raw else ""


class Operator:
    """Base of the operator handles (rc_op)."""

    def __init__(self, ctx: Context, h: C.c_void_p, n: int, complex_: bool):
        self.ctx = ctx
        self.h = h
        self.n = n
        self.complex_ = complex_
        self.dtype = capi.RC_COMPLEX128 if complex_ else capi.RC_REAL64

    def close(self):
        # a destroyed context has already released its operators (rc_ctx_destroy)
        if self.h and self.ctx.h:
            lib().rc_op_destroy(self.h)
        self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def scalar(self):
        return np.complex128 if self.complex_ else np.float64


class CsrOperator(Operator):
    """Hermitian CSR matrix (int32 indices) copied to the device."""

    def __init__(self, ctx: Context, rowptr, colind, vals):
        rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
        colind = np.ascontiguousarray(colind, dtype=np.int32)
        complex_ = np.iscomplexobj(vals)
        vals = np.ascontiguousarray(vals, dtype=np.complex128 if complex_ else np.float64)
        n = rowptr.size - 1
        h = C.c_void_p()
        check(lib().rc_op_csr_create(ctx.h, capi.RC_COMPLEX128 if complex_ else capi.RC_REAL64, n, colind.size,
                                     _ptr(rowptr), _ptr(colind), _ptr(vals), C.byref(h)), ctx.h, "rc_op_csr_create")
        super().__init__(ctx, h, n, complex_)
        self.nnz = colind.size

    @classmethod
    def from_host_pointers(cls, ctx: Context, n: int, nnz: int, rowptr_ptr: int, colind_ptr: int, vals_ptr: int,
                           complex_: bool = False) -> "CsrOperator":
        """Create from host addresses (e.g. pinned torch tensors) without a numpy round trip."""
        h = C.c_void_p()
        check(lib().rc_op_csr_create(ctx.h, capi.RC_COMPLEX128 if complex_ else capi.RC_REAL64, n, nnz,
                                     C.c_void_p(rowptr_ptr), C.c_void_p(colind_ptr), C.c_void_p(vals_ptr),
                                     C.byref(h)), ctx.h, "rc_op_csr_create")
        self = cls.__new__(cls)
        Operator.__init__(self, ctx, h, n, complex_)
        self.nnz = nnz
        return self


    @classmethod
    def from_matrix_market(cls, ctx: Context, path: str) -> "CsrOperator":
        """Create from a Matrix Market coordinate file (read_matrix_market)."""
        rowptr, colind, vals = read_matrix_market(path)
        return cls(ctx, rowptr, colind, vals)


def read_matrix_market(path: str):
    """CSR arrays (rowptr int32, colind int32, vals float64 or complex128) of a square Matrix Market
    'coordinate' file with real, integer or complex entries and general, symmetric or hermitian
    storage. Symmetric and hermitian files store one triangle; the other is filled in (the
    conjugate for hermitian). Duplicate entries are summed; each row's columns come out sorted."""
    with open(path) as f:
        header = f.readline().split()
        if len(header) < 5 or header[0] != "%%MatrixMarket" or header[1].lower() != "matrix":
            raise ValueError(f"{path}: not a Matrix Market matrix file")
        fmt, field, symm = header[2].lower(), header[3].lower(), header[4].lower()
        if fmt != "coordinate":
            raise ValueError(f"{path}: only the coordinate format is supported")
        if field not in ("real", "integer", "complex", "double"):
            raise ValueError(f"{path}: unsupported field {field}")
        if symm not in ("general", "symmetric", "hermitian"):
            raise ValueError(f"{path}: unsupported symmetry {symm}")
        line = f.readline()
        while line.startswith("%") or not line.strip():
            line = f.readline()
        nr, nc, nnz = (int(t) for t in line.split()[:3])
        if nr != nc:
            raise ValueError(f"{path}: the operator must be square ({nr} x {nc})")
        data = np.loadtxt(f, ndmin=2, max_rows=nnz) if nnz > 0 else np.zeros((0, 4))
    if data.shape[0] != nnz:
        raise ValueError(f"{path}: expected {nnz} entries, read {data.shape[0]}")
    i = data[:, 0].astype(np.int64) - 1
    j = data[:, 1].astype(np.int64) - 1
    complex_ = field == "complex"
    v = data[:, 2] + 1j * data[:, 3] if complex_ else data[:, 2].astype(np.float64)
    if symm != "general":
        off = i != j
        vt = np.conj(v[off]) if symm == "hermitian" else v[off]
        i, j, v = np.concatenate([i, j[off]]), np.concatenate([j, i[off]]), np.concatenate([v, vt])
    order = np.lexsort((j, i))
    i, j, v = i[order], j[order], v[order]
    if i.size:  # sum duplicates
        key = i * nr + j
        first = np.concatenate([[True], key[1:] != key[:-1]])
        groups = np.cumsum(first) - 1
        v = np.bincount(groups, weights=v.real, minlength=groups[-1] + 1) + (
            1j * np.bincount(groups, weights=v.imag, minlength=groups[-1] + 1) if complex_ else 0.0)
        i, j = i[first], j[first]
    rowptr = np.zeros(nr + 1, dtype=np.int64)
    np.add.at(rowptr, i + 1, 1)
    rowptr = np.cumsum(rowptr).astype(np.int32)
    return rowptr, j.astype(np.int32), (v.astype(np.complex128) if complex_ else v.astype(np.float64))


class StencilOperator(Operator):
    """Matrix-free 5/7/27-point stencil with a diagonal array (Dirichlet boundaries)."""

    def __init__(self, ctx: Context, kind: int, dims, diag, offdiag: float, flux: float = 0.0,
                 complex_: bool = False):
        dims = tuple(int(d) for d in dims) + (1,) * (3 - len(dims))
        diag = np.ascontiguousarray(diag, dtype=np.float64)
        h = C.c_void_p()
        check(lib().rc_op_stencil_create(ctx.h, capi.RC_COMPLEX128 if complex_ else capi.RC_REAL64, kind, dims[0],
                                         dims[1], dims[2], _ptr(diag), float(offdiag), float(flux), C.byref(h)),
              ctx.h, "rc_op_stencil_create")
        super().__init__(ctx, h, int(np.prod(dims)), complex_)
        self.kind = kind
        self.dims = dims


class CallbackOperator(Operator):
    """Foreign operator: fn(in_ptr, out_ptr, n, s, ld, alpha, beta, stream_ptr) -> int computes
    out = alpha*A*in + beta*out on device column-major blocks (the reference's Otype::apply contract)."""

    def __init__(self, ctx: Context, n: int, fn: Callable, complex_: bool = False):
        def tramp(user, pin, pout, n_, s, ld, alpha, beta, stream):
            try:
                a = complex(alpha[0], alpha[1])
                b = complex(beta[0], beta[1])
                return int(fn(pin, pout, n_, s, ld, a, b, stream) or 0)
            except Exception:  # an exception must not cross the C boundary
                import traceback
                traceback.print_exc()
                return 1

        self._cb = capi.BLOCK_APPLY_FN(tramp)
        h = C.c_void_p()
        check(lib().rc_op_callback_create(ctx.h, capi.RC_COMPLEX128 if complex_ else capi.RC_REAL64, n, self._cb,
                                          None, C.byref(h)), ctx.h, "rc_op_callback_create")
        super().__init__(ctx, h, n, complex_)


def operator_from_problem(ctx: Context, prob, form: str = "csr") -> Operator:
    if form == "stencil":
        return StencilOperator(ctx, prob.kind, prob.dims, prob.diag, prob.offdiag, prob.flux, prob.complex_)
    rp, ci, v = prob.csr()
    return CsrOperator(ctx, rp, ci, v)


class SolveResult:
    def __init__(self, evals, evecs, residuals, info):
        self.evals = evals
        self.evecs = evecs
        self.residuals = residuals
        self.info = info


def make_params(k: int, tol: float, incr: Optional[int] = None, buffer: Optional[int] = None,
                precision: str = "fp64", stop: str = "RESIDUAL_ONLY", **kw) -> capi.SolveParams:
    from .problems import block_sizes
    p = capi.default_params()
    di, db = block_sizes(k)
    p.eig_count = k
    p.tol = tol
    p.subspace_increment = incr if incr is not None else di
    p.buffer_size = buffer if buffer is not None else db
    p.precision = _PREC[precision]
    p.stop_condition = _STOP[stop.upper()]
    for key, val in kw.items():
        setattr(p, key, val)
    return p


def solve(ctx: Context, op: Operator, params: capi.SolveParams, v0=None, host: bool = True, evecs_out=None,
          want_vectors: bool = True) -> SolveResult:
    """Run rc_solve. host=True: v0 / eigenvectors are host numpy arrays (column-major, returned as
    an (found, n) C-ordered array whose row j is eigenvector j). host=False: v0 and evecs_out are
    device pointers/tensors."""
    k = int(params.eig_count if params.mode in (0, 1) else max(params.eig_count, 1))
    params.host_buffers = 1 if host else 0
    keep = []
    if v0 is not None:
        params.non_random_start = 1
        if host and not isinstance(v0, int):
            v0 = np.ascontiguousarray(v0, dtype=op.scalar)
            keep.append(v0)
            params.v0_cols = v0.shape[0] if v0.ndim == 2 else 1
        elif params.v0_cols <= 0:
            params.v0_cols = int(params.subspace_increment + params.buffer_size)
    evals = np.zeros(max(k, 1), dtype=np.float64)
    resid = np.zeros(max(k, 1), dtype=np.float64)
    if evecs_out is not None:
        evecs = evecs_out
    elif want_vectors and host:
        evecs = np.zeros((max(k, 1), op.n), dtype=op.scalar)
    else:
        evecs = None
    info = capi.SolveInfo()
    info.struct_size = C.sizeof(capi.SolveInfo)
    params.struct_size = C.sizeof(capi.SolveParams)
    check(lib().rc_solve(ctx.h, op.h, C.byref(params), C.c_void_p(_ptr(v0)),
                         evals.ctypes.data_as(C.POINTER(C.c_double)), C.c_void_p(_ptr(evecs)),
                         resid.ctypes.data_as(C.POINTER(C.c_double)), C.byref(info)), ctx.h, "rc_solve")
    f = info.found
    ev = evecs[:f] if isinstance(evecs, np.ndarray) else evecs
    return SolveResult(evals[:f].copy(), ev, resid[:f].copy(), info.as_dict())


# ---- request server (rc_server_*, rc_serve_*) ---------------------------------------------------
class Request:
    """One submitted solve. The server writes the eigenvalues, residuals and (host) eigenvectors
    into the arrays held here when the request finishes."""

    def __init__(self, server: "Server", rid: int, op: Operator, evals, resid, evecs, keep):
        self.server = server
        self.id = rid
        self.op = op
        self._evals = evals
        self._resid = resid
        self._evecs = evecs
        self._keep = keep

    def state(self) -> str:
        st = C.c_int()
        self.server._check(lib().rc_serve_poll(self.server.h, self.id, C.byref(st)), "rc_serve_poll")
        return capi.REQ_STATE_NAMES[st.value]

    def wait(self, timeout_ms: float = -1.0) -> str:
        """Block until the request finishes (or timeout_ms passes); returns its state."""
        st = C.c_int()
        rc = lib().rc_serve_wait(self.server.h, self.id, float(timeout_ms), C.byref(st))
        if rc not in (capi.RC_OK, 10):
            self.server._check(rc, "rc_serve_wait")
        return capi.REQ_STATE_NAMES[st.value]

    def cancel(self):
        self.server._check(lib().rc_serve_cancel(self.server.h, self.id), "rc_serve_cancel")

    def info(self) -> dict:
        """Timings and memory of the request (rc_request_info), available in every state."""
        ri = capi.RequestInfo()
        ri.struct_size = C.sizeof(capi.RequestInfo)
        lib().rc_serve_result(self.server.h, self.id, None, C.byref(ri), None, 0)
        return ri.as_dict()

    def result(self) -> SolveResult:
        """The finished solve; raises RCError with the request's own status when it failed."""
        info = capi.SolveInfo()
        info.struct_size = C.sizeof(capi.SolveInfo)
        ri = capi.RequestInfo()
        ri.struct_size = C.sizeof(capi.RequestInfo)
        err = C.create_string_buffer(512)
        rc = lib().rc_serve_result(self.server.h, self.id, C.byref(info), C.byref(ri), err, 512)
        if rc != capi.RC_OK:
            raise capi.RCError(rc, err.value.decode())
        f = info.found
        ev = self._evecs[:f] if isinstance(self._evecs, np.ndarray) else self._evecs
        d = info.as_dict()
        d["request"] = ri.as_dict()
        return SolveResult(self._evals[:f].copy(), ev, self._resid[:f].copy(), d)

    def release(self):
        self.server._check(lib().rc_serve_release(self.server.h, self.id), "rc_serve_release")


class Server:
    """Continuous-batching eigen-solve server on one GPU (rc_server)."""

    def __init__(self, device: int = 0, budget_bytes: int = 0, max_active: int = 16, batch_window_us: float = 200.0,
                 use_graphs: bool = True, starvation_ms: float = 2000.0):
        p = capi.ServerParams()
        lib().rc_server_params_default(C.byref(p))
        p.device = device
        p.hbm_budget_bytes = int(budget_bytes)
        p.max_active = int(max_active)
        p.batch_window_us = float(batch_window_us)
        p.use_graphs = 1 if use_graphs else 0
        p.starvation_ms = float(starvation_ms)
        self.h = C.c_void_p()
        check(lib().rc_server_create(C.byref(p), C.byref(self.h)), None, "rc_server_create")

    def _check(self, rc: int, what: str):
        if rc != capi.RC_OK:
            raw = lib().rc_server_last_error(self.h) if self.h else b""
            raise capi.RCError(rc, f"{what}: {raw.decode() if raw else ''}")

    def submit(self, op: Operator, params: capi.SolveParams, v0=None, want_vectors: bool = True) -> Request:
        """Queue a solve; v0 and the eigenvectors are host numpy arrays (column-major blocks, given
        and returned as (columns, n) C-ordered arrays)."""
        k = int(params.eig_count if params.mode in (0, 1) else max(params.eig_count, 1))
        params.host_buffers = 1
        keep = [params]
        if v0 is not None:
            v0 = np.ascontiguousarray(v0, dtype=op.scalar)
            keep.append(v0)
            params.non_random_start = 1
            params.v0_cols = v0.shape[0] if v0.ndim == 2 else 1
        evals = np.zeros(max(k, 1), dtype=np.float64)
        resid = np.zeros(max(k, 1), dtype=np.float64)
        evecs = np.zeros((max(k, 1), op.n), dtype=op.scalar) if want_vectors else None
        params.struct_size = C.sizeof(capi.SolveParams)
        rid = C.c_int64()
        self._check(lib().rc_serve_submit(self.h, op.h, C.byref(params), C.c_void_p(_ptr(v0)),
                                          evals.ctypes.data_as(C.POINTER(C.c_double)), C.c_void_p(_ptr(evecs)),
                                          resid.ctypes.data_as(C.POINTER(C.c_double)), C.byref(rid)),
                    "rc_serve_submit")
        return Request(self, rid.value, op, evals, resid, evecs, keep)

    def stats(self) -> dict:
        st = capi.ServerStats()
        st.struct_size = C.sizeof(capi.ServerStats)
        self._check(lib().rc_server_stats_get(self.h, C.byref(st)), "rc_server_stats_get")
        return st.as_dict()

    def close(self):
        if self.h:
            lib().rc_server_destroy(self.h)
            self.h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- kernel-level calls -------------------------------------------------------------------
def spmm(ctx: Context, op: Operator, X, Y, s: int, alpha=1.0, beta=0.0, ldx=None, ldy=None):
    a = (C.c_double * 2)(complex(alpha).real, complex(alpha).imag)
    b = (C.c_double * 2)(complex(beta).real, complex(beta).imag)
    check(lib().rc_spmm(ctx.h, op.h, C.c_void_p(_ptr(X)), ldx or op.n, C.c_void_p(_ptr(Y)), ldy or op.n, s, a, b),
          ctx.h, "rc_spmm")


def filter_block(ctx: Context, op: Operator, X, s: int, degree: int, gamma1: float, gamma2: float,
                 precision: str = "fp64", repetition: int = 1, ld=None):
    check(lib().rc_filter(ctx.h, op.h, C.c_void_p(_ptr(X)), ld or op.n, s, degree, repetition, gamma1, gamma2,
                          _PREC[precision]), ctx.h, "rc_filter")


def rm_leading_dim(complex_: bool, precision: str, s: int) -> int:
    """Leading dimension of the filter's row-major blocks (rc_rm_leading_dim)."""
    return int(lib().rc_rm_leading_dim(capi.RC_COMPLEX128 if complex_ else capi.RC_REAL64, _PREC[precision], s))


def filter_step_rm(ctx: Context, op: Operator, x, z, y, s: int, alpha, beta, gamma=0.0, precision: str = "fp64",
                   ld=None):
    """One degree step y = alpha A x + beta x + gamma z on row-major device blocks (rc_filter_step_rm)."""
    def pair(v):
        v = complex(v)
        return (C.c_double * 2)(v.real, v.imag)
    ld = ld or rm_leading_dim(op.complex_, precision, s)
    check(lib().rc_filter_step_rm(ctx.h, op.h, C.c_void_p(_ptr(x)), C.c_void_p(_ptr(z)), C.c_void_p(_ptr(y)), ld, s,
                                  pair(alpha), pair(beta), pair(gamma), _PREC[precision]), ctx.h,
          "rc_filter_step_rm")


def filter_correction(ctx: Context, op: Operator, V, s: int, lam, degree: int, gamma1: float, gamma2: float,
                      ld=None):
    """V <- P_m(A')V in correction form on Ritz pairs (V, lam): rc_filter_correction."""
    lam = np.ascontiguousarray(lam, dtype=np.float64)
    check(lib().rc_filter_correction(ctx.h, op.h, C.c_void_p(_ptr(V)), ld or op.n, s,
                                     lam.ctypes.data_as(capi.c_dp), degree, gamma1, gamma2),
          ctx.h, "rc_filter_correction")


def filter_correction_batch(ctx: Context, jobs) -> int:
    """Several correction-filter applications in one batched launch per degree step
    (rc_filter_correction_batch). jobs: (op, V, s, lam, degree, gamma1, gamma2) tuples.
    Returns the number of jobs that ran in the batched launches."""
    arr = (capi.CorrectionJob * len(jobs))()
    keep = []
    for j, (op, V, s, lam, degree, g1, g2) in enumerate(jobs):
        lam = np.ascontiguousarray(lam, dtype=np.float64)
        keep.append(lam)
        arr[j] = capi.CorrectionJob(C.sizeof(capi.CorrectionJob), op.h, _ptr(V), op.n, s, int(lam.ctypes.data),
                                    degree, g1, g2)
    batched = C.c_int()
    check(lib().rc_filter_correction_batch(ctx.h, len(jobs), arr, C.byref(batched)), ctx.h,
          "rc_filter_correction_batch")
    return batched.value


def lanczos_bounds(ctx: Context, op: Operator, v0=None, seed: int = 1, tol: float = 1e-6, which: str = "max",
                   max_iter: int = 10000):
    lmin, lmax, it = C.c_double(), C.c_double(), C.c_int64()
    keep = None
    if v0 is not None:
        keep = np.ascontiguousarray(v0, dtype=op.scalar)
    w = {"both": 0, "max": 1, "min": 2}[which]
    check(lib().rc_lanczos_bounds(ctx.h, op.h, C.c_void_p(_ptr(keep)), seed, tol, w, max_iter, C.byref(lmin),
                                  C.byref(lmax), C.byref(it)), ctx.h, "rc_lanczos_bounds")
    return lmin.value, lmax.value, it.value


def cholqr(ctx: Context, V, n: int, s: int, complex_: bool = False, ld=None) -> int:
    passes = C.c_int()
    check(lib().rc_cholqr(ctx.h, capi.RC_COMPLEX128 if complex_ else capi.RC_REAL64, C.c_void_p(_ptr(V)), ld or n,
                          n, s, C.byref(passes)), ctx.h, "rc_cholqr")
    return passes.value


def rayleigh_ritz(ctx: Context, op: Operator, V, W, s: int, res_count: int, ld=None):
    evals = np.zeros(s)
    res = np.zeros(max(res_count, 1))
    Q = np.zeros((s, s), dtype=op.scalar)
    check(lib().rc_rayleigh_ritz(ctx.h, op.h, C.c_void_p(_ptr(V)), C.c_void_p(_ptr(W)), ld or op.n, s, res_count,
                                 evals.ctypes.data_as(C.POINTER(C.c_double)),
                                 res.ctypes.data_as(C.POINTER(C.c_double)), C.c_void_p(_ptr(Q))), ctx.h,
          "rc_rayleigh_ritz")
    return evals, res[:res_count], Q.T.copy()  # Q returned column-major -> transpose to row-major


def small_eigh(ctx: Context, H: np.ndarray):
    """Eigen-decomposition of a small Hermitian matrix on the GPU. Returns (evals, Q) with Q's
    columns the eigenvectors."""
    complex_ = np.iscomplexobj(H)
    s = H.shape[0]
    Hc = np.asfortranarray(H, dtype=np.complex128 if complex_ else np.float64)
    evals = np.zeros(s)
    Q = np.zeros((s, s), dtype=Hc.dtype, order="F")
    check(lib().rc_small_eigh(ctx.h, capi.RC_COMPLEX128 if complex_ else capi.RC_REAL64, s, C.c_void_p(_ptr(Hc)),
                              evals.ctypes.data_as(C.POINTER(C.c_double)), C.c_void_p(_ptr(Q))), ctx.h,
          "rc_small_eigh")
    return evals, Q


# ---- host-only polynomial design ------------------------------------------------------------
def cpoly_xstar(m: int):
    x, u = C.c_double(), C.c_double()
    check(lib().rc_cpoly_xstar(m, C.byref(x), C.byref(u)))
    return x.value, u.value


def cpoly_star_degree(shift: float, lambda_bound: float, lambda_star: float, degree_max: int = 200):
    d, b = C.c_int64(), C.c_double()
    check(lib().rc_cpoly_star_degree(shift, lambda_bound, lambda_star, degree_max, C.byref(d), C.byref(b)))
    return d.value, b.value


def cpoly_gammas(m: int, lambda_max: float, shift: float):
    g1, g2 = C.c_double(), C.c_double()
    check(lib().rc_cpoly_gammas(m, lambda_max, shift, C.byref(g1), C.byref(g2)))
    return g1.value, g2.value
