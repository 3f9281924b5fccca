"""Residuals of returned eigenpairs recomputed outside the library's kernels.

A caller (or a benchmark) that wants to check a solve without trusting the library's own operator
apply writes the operator out in plain torch arithmetic: the Dirichlet stencils of the synthetic
workloads on their grid (stencil_apply), or torch's sparse CSR product for a CSR matrix
(csr_residuals). Both work on the GPU in FP64 / c128.
"""
from __future__ import annotations

import numpy as np


def stencil_apply(P, X):
    """A X for the rows of X (k x n), the Dirichlet stencil of problem P in torch arithmetic: diag * x
    plus offdiag times every neighbour on the grid (zero padding at the boundary); for complex P the
    y-bonds carry exp(+i 2 pi flux x) from (x, y-1) and its conjugate from (x, y+1)."""
    import torch
    k = X.shape[0]
    nx, ny, nz = P.nx, P.ny, P.nz
    Xg = X.reshape(k, nz, ny, nx)
    pad = (1, 1, 1, 1, 1, 1)
    if X.is_complex():
        Xp = torch.complex(torch.nn.functional.pad(Xg.real, pad), torch.nn.functional.pad(Xg.imag, pad))
    else:
        Xp = torch.nn.functional.pad(Xg, pad)
    diag = torch.from_numpy(P.diag).to(X.device).reshape(nz, ny, nx)
    out = Xg * diag
    if P.kind == 27:
        offs = [(dz, dy, dx) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1) if (dz, dy, dx) != (0, 0, 0)]
    else:
        offs = [(-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1)]
    for dz, dy, dx in offs:
        nb = Xp[:, 1 + dz:1 + dz + nz, 1 + dy:1 + dy + ny, 1 + dx:1 + dx + nx]
        if X.is_complex() and dy != 0 and dx == 0 and dz == 0:
            th = 2.0 * np.pi * P.flux * torch.arange(nx, device=X.device, dtype=torch.float64)
            ph = torch.polar(torch.ones_like(th), th if dy < 0 else -th)
            nb = nb * ph
        out = out + P.offdiag * nb
    return out.reshape(k, -1)


def stencil_residuals(P, X, evals, chunk: int = 8) -> np.ndarray:
    """||A x_j - lam_j x_j|| / max(|lam_j|, 0.1) (the stop test's relative residual) for the rows x_j
    of X (k x n, device), a few rows at a time so the padded grid copies stay small."""
    import torch
    k = X.shape[0]
    rel = np.empty(k)
    with torch.no_grad():
        for c0 in range(0, k, chunk):
            Xc = X[c0:c0 + chunk]
            lam = torch.from_numpy(np.asarray(evals[c0:c0 + chunk], dtype=np.float64)).to(X.device)
            if X.is_complex():
                lam = lam.to(X.dtype)
            r = torch.linalg.vector_norm(stencil_apply(P, Xc) - lam[:, None] * Xc, dim=1).cpu().numpy()
            rel[c0:c0 + chunk] = r / np.maximum(np.abs(evals[c0:c0 + chunk]), 0.1)
    return rel
