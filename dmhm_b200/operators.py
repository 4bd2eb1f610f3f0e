"""Grid operators of the H-matrix workloads, as hierarchical-order CSR.

The reference's drivers build these by hand row by row (FormRow in
tests/HMat2d/Invert.cpp:14-67 and :140-181); this module builds the same kind
of matrix vectorised:

* ``stencil(sizes, coef, num_levels)``: 5-point (2-D) or 7-point (3-D)
  variable-coefficient operator with diagonal ``2*d*c_i + shift`` and
  off-diagonals ``-min(c_i, c_j)`` (symmetric positive definite for c > 0),
  each row ordered x-1, x+1, y-1, y+1[, z-1, z+1], diagonal;
* coefficient fields: uniform in [1, 2) or log-uniform in [1, 100) from a
  seeded numpy generator.

All vectors are permuted into the hierarchical ordering of
BuildNaturalToHierarchicalMap so they can be handed to an H-matrix directly.
"""
from __future__ import annotations

from typing import Sequence

import numpy as np

from .hmat import Sparse, natural_to_hierarchical_map


def uniform_coefficients(sizes: Sequence[int], seed: int) -> np.ndarray:
    """c ~ U[1, 2) per cell, natural order."""
    rng = np.random.default_rng(seed)
    return 1.0 + rng.random(int(np.prod(sizes)))


def log_uniform_coefficients(sizes: Sequence[int], seed: int, lo=1.0, hi=100.0) -> np.ndarray:
    """c log-uniform in [lo, hi) per cell, natural order."""
    rng = np.random.default_rng(seed)
    return lo * (hi / lo) ** rng.random(int(np.prod(sizes)))


def stencil(sizes: Sequence[int], coef: np.ndarray, num_levels: int,
            shift: float = 0.1) -> Sparse:
    sizes = [int(s) for s in sizes]
    d = len(sizes)
    N = int(np.prod(sizes))
    mp = natural_to_hierarchical_map(sizes, num_levels).astype(np.int64)
    inv = np.empty(N, dtype=np.int64)
    inv[mp] = np.arange(N)
    nat = inv                       # natural index of each hierarchical row
    nx = sizes[0]
    ny = sizes[1]
    x = nat % nx
    y = (nat // nx) % ny
    z = nat // (nx * ny)
    cand = [(x > 0, -1), (x < nx - 1, 1), (y > 0, -nx), (y < ny - 1, nx)]
    if d == 3:
        nz = sizes[2]
        cand += [(z > 0, -nx * ny), (z < nz - 1, nx * ny)]
    ci = coef[nat]
    cols = np.full((N, len(cand) + 1), -1, dtype=np.int64)
    vals = np.zeros((N, len(cand) + 1))
    for k, (mask, step) in enumerate(cand):
        nb = nat + step
        cols[mask, k] = mp[nb[mask]]
        vals[mask, k] = -np.minimum(ci[mask], coef[nb[mask]])
    cols[:, -1] = mp[nat]
    vals[:, -1] = 2.0 * d * ci + shift
    keep = cols >= 0
    counts = keep.sum(axis=1)
    rows = np.zeros(N + 1, dtype=np.int64)
    np.cumsum(counts, out=rows[1:])
    return Sparse(N, N, rows, cols[keep].astype(np.int32), vals[keep])


def to_hierarchical(v_natural: np.ndarray, sizes: Sequence[int], num_levels: int) -> np.ndarray:
    """Permute a natural-order vector (or the rows of a matrix) into
    hierarchical order."""
    mp = natural_to_hierarchical_map(sizes, num_levels)
    out = np.empty_like(v_natural)
    out[mp] = v_natural
    return out


def helmholtz(sizes: Sequence[int], wavenumber: float, num_levels: int,
              absorption: float = 0.2) -> Sparse:
    """Shifted five-point (2-D) or seven-point (3-D) Helmholtz-like operator,
    complex: diagonal 2 d + absorption i - (k h)^2 with h = 1 / (side + 1) of
    the first axis, off-diagonals -1; CSR in hierarchical order with complex
    nonzeros (HMat2d<std::complex<double>> input)."""
    sizes = [int(s) for s in sizes]
    d = len(sizes)
    N = int(np.prod(sizes))
    mp = natural_to_hierarchical_map(sizes, num_levels).astype(np.int64)
    inv = np.empty(N, dtype=np.int64)
    inv[mp] = np.arange(N)
    nat = inv
    nx, ny = sizes[0], sizes[1]
    x = nat % nx
    y = (nat // nx) % ny
    z = nat // (nx * ny)
    cand = [(x > 0, -1), (x < nx - 1, 1), (y > 0, -nx), (y < ny - 1, nx)]
    if d == 3:
        nz = sizes[2]
        cand += [(z > 0, -nx * ny), (z < nz - 1, nx * ny)]
    h = 1.0 / (sizes[0] + 1)
    cols = np.full((N, len(cand) + 1), -1, dtype=np.int64)
    vals = np.zeros((N, len(cand) + 1), dtype=np.complex128)
    for k, (mask, step) in enumerate(cand):
        nb = nat + step
        cols[mask, k] = mp[nb[mask]]
        vals[mask, k] = -1.0
    cols[:, -1] = mp[nat]
    vals[:, -1] = 2.0 * d + 1j * absorption - (wavenumber * h) ** 2
    keep = cols >= 0
    counts = keep.sum(axis=1)
    rows = np.zeros(N + 1, dtype=np.int64)
    np.cumsum(counts, out=rows[1:])
    return Sparse(N, N, rows, cols[keep].astype(np.int32), vals[keep])


def dense_from_sparse(S: Sparse) -> np.ndarray:
    """Dense copy of a CSR matrix (small sizes; test and check use)."""
    A = np.zeros((S.height, S.width), dtype=np.asarray(S.nonzeros).dtype)
    for i in range(S.height):
        for k in range(int(S.rowOffsets[i]), int(S.rowOffsets[i + 1])):
            A[i, int(S.columnIndices[k])] += S.nonzeros[k]
    return A
