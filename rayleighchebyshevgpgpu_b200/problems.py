"""Synthetic operators and start blocks for the benchmark configurations.

The reference ships no operators or datasets; these are the seeded synthetic Hamiltonians the
benchmark configurations name. Grid index i = x + nx*(y + ny*z); Dirichlet boundaries.

  config 1  2D 5-point Laplacian 64x64 + V~U[0,1) (seed 0); k=16, tol 1e-10, start N(0,1) seed 1
  config 2  3D 7-point Laplacian 128^3 + V~U[0,4) (seed 2); k=64, tol 1e-10, start N(0,1) seed 3
  config 3  3D tight binding 96^3, hopping -1 with Peierls phase exp(+i 2 pi phi x) on y-bonds
            (Landau gauge, flux phi=1/17 along z), on-site V~U[-1,1) (seed 4); k=128, tol 1e-9,
            complex start N(0,1)+iN(0,1) from seed 40
  config 5  3D 27-point stencil 256^3, off-diagonal -1/26, diagonal 1+V, V~U[0,2) (seed 6);
            k=32, tol 1e-10, start N(0,1) seed 7

Block size convention: incr = k, buffer = max(8, k/2) rounded up to a multiple of 8.
Start blocks are column-major n x s: column j holds draws j*n .. (j+1)*n-1 of the generator.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


def block_sizes(k: int) -> tuple[int, int]:
    buf = max(8, k // 2)
    buf = ((buf + 7) // 8) * 8
    return k, buf


@dataclass
class Problem:
    name: str
    dims: tuple
    kind: int                      # 5, 7 or 27 (stencil form)
    diag: np.ndarray               # float64, length n (full diagonal incl. constant)
    offdiag: float
    flux: float = 0.0
    complex_: bool = False
    k: int = 16
    tol: float = 1e-10
    start_seed: int = 1
    meta: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return int(np.prod(self.dims))

    @property
    def nx(self):
        return self.dims[0]

    @property
    def ny(self):
        return self.dims[1] if len(self.dims) > 1 else 1

    @property
    def nz(self):
        return self.dims[2] if len(self.dims) > 2 else 1

    def csr(self):
        return stencil_csr(self.dims, self.kind, self.diag, self.offdiag, self.flux, self.complex_)

    def start_block(self, s: int) -> np.ndarray:
        """Column-major start block as a C-ordered (s, n) array (row j = column j)."""
        rng = np.random.default_rng(self.start_seed)
        if self.complex_:
            re = rng.standard_normal((s, self.n))
            im = rng.standard_normal((s, self.n))
            return re + 1j * im
        return rng.standard_normal((s, self.n))


def stencil_csr(dims, kind: int, diag: np.ndarray, offdiag: float, flux: float = 0.0, complex_: bool = False):
    """CSR (rowptr int32, colind int32, vals float64/complex128) with sorted columns."""
    dims = tuple(int(d) for d in dims)
    nx = dims[0]
    ny = dims[1] if len(dims) > 1 else 1
    nz = dims[2] if len(dims) > 2 else 1
    n = nx * ny * nz
    idx = np.arange(n, dtype=np.int64)
    ix = idx % nx
    iy = (idx // nx) % ny
    iz = idx // (nx * ny)
    if kind == 27:
        offs = [(dx, dy, dz) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]
    elif kind == 7:
        offs = [(0, 0, -1), (0, -1, 0), (-1, 0, 0), (0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1)]
    elif kind == 5:
        offs = [(0, -1, 0), (-1, 0, 0), (0, 0, 0), (1, 0, 0), (0, 1, 0)]
    else:
        raise ValueError("kind must be 5, 7 or 27")
    masks = []
    for dx, dy, dz in offs:
        m = np.ones(n, dtype=bool)
        if dx < 0: m &= ix > 0
        if dx > 0: m &= ix < nx - 1
        if dy < 0: m &= iy > 0
        if dy > 0: m &= iy < ny - 1
        if dz < 0: m &= iz > 0
        if dz > 0: m &= iz < nz - 1
        masks.append(m)
    counts = np.zeros(n, dtype=np.int64)
    for m in masks:
        counts += m
    rowptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=rowptr[1:])
    nnz = int(rowptr[-1])
    colind = np.empty(nnz, dtype=np.int32)
    vals = np.empty(nnz, dtype=np.complex128 if complex_ else np.float64)
    cursor = rowptr[:-1].copy()
    theta = 2.0 * np.pi * flux
    for (dx, dy, dz), m in zip(offs, masks):
        rows = idx[m]
        pos = cursor[m]
        colind[pos] = (rows + dx + dy * nx + dz * nx * ny).astype(np.int32)
        if (dx, dy, dz) == (0, 0, 0):
            vals[pos] = diag[m]
        elif complex_ and dy != 0 and dx == 0 and dz == 0:
            ph = np.exp((1j if dy < 0 else -1j) * theta * ix[m])
            vals[pos] = offdiag * ph
        else:
            vals[pos] = offdiag
        cursor[m] += 1
    return rowptr.astype(np.int32), colind, vals


def config1() -> Problem:
    n = 64 * 64
    V = np.random.default_rng(0).uniform(0.0, 1.0, n)
    return Problem("config1_2d5pt_64x64", (64, 64), 5, 4.0 + V, -1.0, k=16, tol=1e-10, start_seed=1)


def config2(side: int = 128) -> Problem:
    n = side ** 3
    V = np.random.default_rng(2).uniform(0.0, 4.0, n)
    return Problem(f"config2_3d7pt_{side}^3", (side, side, side), 7, 6.0 + V, -1.0, k=64, tol=1e-10,
                   start_seed=3)


def config3(side: int = 96, k: int = 128) -> Problem:
    n = side ** 3
    V = np.random.default_rng(4).uniform(-1.0, 1.0, n)
    return Problem(f"config3_tb_{side}^3_phi1/17", (side, side, side), 7, V, -1.0, flux=1.0 / 17.0,
                   complex_=True, k=k, tol=1e-9, start_seed=40)


def config5(side: int = 256) -> Problem:
    n = side ** 3
    V = np.random.default_rng(6).uniform(0.0, 2.0, n)
    return Problem(f"config5_3d27pt_{side}^3", (side, side, side), 27, 1.0 + V, -1.0 / 26.0, k=32, tol=1e-10,
                   start_seed=7)


def small_laplacian(dims, seed: int = 0, vmax: float = 1.0, k: int = 8, complex_: bool = False,
                    flux: float = 0.0) -> Problem:
    """Small random-potential Laplacian (tests)."""
    n = int(np.prod(dims))
    rng = np.random.default_rng(seed)
    if complex_:
        V = rng.uniform(-1.0, 1.0, n)
        return Problem(f"tb{dims}", tuple(dims), 7 if len(dims) == 3 else 5, V, -1.0, flux=flux, complex_=True,
                       k=k, start_seed=seed + 100)
    V = rng.uniform(0.0, vmax, n)
    kind = {1: 5, 2: 5, 3: 7}[len(dims)]
    d0 = 2.0 * len(dims)
    if len(dims) == 1:
        dims = (dims[0], 1)
    return Problem(f"lap{dims}", tuple(dims), kind, d0 + V, -1.0, k=k, start_seed=seed + 100)


@dataclass
class ServeRequest:
    """One request of the serving stream: its operator, eigenpair count, tolerance and arrival."""
    index: int
    problem: Problem
    arrival_gap: float   # unit-rate exponential gap before this arrival (scale by 1/rate)


def serve_stream(count: int = 256, seed: int = 5, nmin: float = 1e4, nmax: float = 2e6) -> list:
    """Configuration 4: a Poisson stream of random-potential Laplacians.

    Each request draws, from one generator seeded with `seed`: the operator (2D 5-point or 3D
    7-point, equal odds), n log-uniform in [nmin, nmax] (grid side round(n^(1/d))), the disorder
    W ~ U[1, 8], k from {8, 16, 32, 64} and tol from {1e-8, 1e-10}, and a unit-rate exponential
    arrival gap. Its potential V ~ U[0, W) comes from its own generator seeded (seed, index).
    """
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        kind = 5 if rng.random() < 0.5 else 7
        n_target = float(np.exp(rng.uniform(np.log(nmin), np.log(nmax))))
        W = float(rng.uniform(1.0, 8.0))
        k = int(rng.choice([8, 16, 32, 64]))
        tol = float(rng.choice([1e-8, 1e-10]))
        gap = float(rng.exponential(1.0))
        d = 2 if kind == 5 else 3
        side = max(2, int(round(n_target ** (1.0 / d))))
        dims = (side, side) if d == 2 else (side, side, side)
        n = int(np.prod(dims))
        V = np.random.default_rng([seed, i]).uniform(0.0, W, n)
        P = Problem(f"serve{i}_{d}d{kind}pt_{side}", dims, kind, 2.0 * d + V, -1.0, k=k, tol=tol,
                    start_seed=1000 + i, meta={"W": W})
        out.append(ServeRequest(i, P, gap))
    return out
