"""rc_small_eigh_noalloc: the small Hermitian eigensolver for callers that cannot allocate device
memory (code under a fixed device-memory budget, or a callback of another library's allocator or
operator apply(), where allocating would re-enter that library). Its device staging and work memory
is one fixed array of the library instead of the context's allocator. Checked through the C ABI
against rc_small_eigh, the allocating entry point, on two calls in a row (the second reuses the
array the first one left behind).

This file sorts last so that a run stopping at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from rayleighchebyshevgpgpu_b200 import _capi

pytestmark = pytest.mark.gpu


def _call(fn, ctx, H):
    complex_ = np.iscomplexobj(H)
    s = H.shape[0]
    Hc = np.asfortranarray(H, dtype=np.complex128 if complex_ else np.float64)
    evals = np.zeros(s)
    Q = np.zeros((s, s), dtype=Hc.dtype, order="F")
    st = fn(ctx.h, _capi.RC_COMPLEX128 if complex_ else _capi.RC_REAL64, s, Hc.ctypes.data,
            evals.ctypes.data_as(C.POINTER(C.c_double)), Q.ctypes.data)
    return st, evals, Q


def _hermitian(rng, s, complex_):
    H = rng.standard_normal((s, s))
    if complex_:
        H = H + 1j * rng.standard_normal((s, s))
    return H + H.conj().T


def test_noalloc_matches_allocating_entry_point_two_calls(ctx):
    L = _capi.lib()
    rng = np.random.default_rng(2024)
    # two calls in a row: a real block that does not fit in shared memory, then a complex one
    for s, complex_ in ((128, False), (120, True)):
        H = _hermitian(rng, s, complex_)
        st_ref, ev_ref, Q_ref = _call(L.rc_small_eigh, ctx, H)
        st, ev, Q = _call(L.rc_small_eigh_noalloc, ctx, H)
        assert st_ref == 0 and st == 0, ctx.last_error()
        nrm = np.abs(ev_ref).max()
        # the same tolerance as the allocating solver's own tests (test_small_eigh_matches_lapack)
        assert np.abs(ev - ev_ref).max() < 1e-13 * nrm * s
        assert np.abs(Q.conj().T @ Q - np.eye(s)).max() < 1e-12 * s
        assert np.abs(H @ Q - Q * ev).max() < 1e-12 * nrm * s
        # same eigenvectors up to a phase (the spectrum of a random matrix is simple)
        overlap = np.abs(np.diag(Q_ref.conj().T @ Q))
        assert np.abs(overlap - 1.0).max() < 1e-9


def test_noalloc_allocates_no_device_memory(ctx):
    """After one set-up call, further calls change neither the context's device memory (its
    scratch slots and operator copies) nor the device's free memory; the grid-form Jacobi that a
    block of this width takes (working copies in global memory) runs on the library's array."""
    import torch
    L = _capi.lib()
    rng = np.random.default_rng(7)
    H1, H2 = _hermitian(rng, 128, False), _hermitian(rng, 110, True)
    assert _call(L.rc_small_eigh_noalloc, ctx, H1)[0] == 0  # set-up call
    torch.cuda.synchronize()
    slots0 = ctx.device_bytes()
    free0 = torch.cuda.mem_get_info()[0]
    for H in (H1, H2, H1):
        st, ev, Q = _call(L.rc_small_eigh_noalloc, ctx, H)
        assert st == 0, ctx.last_error()
        assert np.abs(ev - np.linalg.eigvalsh(H)).max() < 1e-13 * np.abs(ev).max() * H.shape[0]
    torch.cuda.synchronize()
    assert ctx.device_bytes() == slots0
    assert torch.cuda.mem_get_info()[0] == free0


def test_noalloc_rejects_sizes_beyond_its_array(ctx):
    L = _capi.lib()
    H = _hermitian(np.random.default_rng(1), 129, False)
    st, _, _ = _call(L.rc_small_eigh_noalloc, ctx, H)
    assert st == 1  # RC_ERR_INVALID
    assert "128" in ctx.last_error()
