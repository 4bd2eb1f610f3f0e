"""CPU restatement of the engine's rounding operation.

TEST INFRASTRUCTURE ONLY.  Nothing in the product imports this module; only
``tests/`` use it, as the checker.

The reference rounds a sum of low-rank terms with LAPACK: QR of the stacked
factors (?geqrf), the SVD of the small core (?gesvd) and the truncation to
maxRank or to the compression tolerance (src/hmat_tools/RoundedUpdate.cpp
:14-162, src/DistHMat2d/Truncation-incl.hpp:37-63).  The engine's rounding
kernel (``round_worker_kernel`` in dmhm_b200/csrc/lowrank.cu) keeps the QR
and the truncation but replaces ?gesvd by a one-sided Jacobi SVD of the core
-- Hestenes' method (M. R. Hestenes, J. SIAM 6, 1958) with the round-robin
pair ordering of Brent and Luk (SIAM J. Sci. Stat. Comput. 6, 1985), one
parallel convergence test over all column pairs before each sweep, and a
bounded number of sweeps.  This module restates that algorithm step by step
in numpy (float64, or float32 for the low-precision phase) so that it can be
checked against LAPACK on the CPU; the GPU kernel's own results are checked
against the reference's LAPACK rounding through the oracle in
``dmhm_oracle.py``.
"""
from __future__ import annotations

import math

import numpy as np
import scipy.linalg as sla

SWEEPS = 40                                    # kJacobiSweeps
JTOL = {np.float64: 1e-15, np.float32: 1e-6}   # Prec<R>::jtol
TINY = {np.float64: 1e-32, np.float32: 1e-12}  # Prec<R>::tiny (relative to ||M||_F^2)


def rr_pos(i: int, step: int, n: int) -> int:
    """Round-robin position: in step `step` the pairs are
    (rr_pos(k), rr_pos(n - 1 - k)) for k < n / 2; position 0 stays, the
    others rotate, so every pair meets once in n - 1 steps."""
    return 0 if i == 0 else 1 + (i - 1 + step) % (n - 1)


def jacobi(M: np.ndarray, dtype=np.float64, all_pairs_test: bool = True):
    """One-sided Jacobi on the columns of M (rows x cols).

    Returns (M_out, J, sweeps): M_out has mutually orthogonal columns, J is
    the accumulated rotation (orthogonal, cols x cols) with M = M_out J^T,
    and sweeps the number of sweeps run.  A pair (p, q) rotates when both
    squared column norms exceed tiny = TINY * ||M||_F^2 and its inner
    product c has c^2 > JTOL^2 a b; the rotation's tangent is the smaller
    root of t^2 + 2 zeta t - 1 = 0, zeta = (b - a) / (2 c), and the squared
    norms are updated as a - t c and b + t c.  With `all_pairs_test` a sweep
    runs only if some pair would rotate at its start."""
    M = np.array(M, dtype=dtype, copy=True)
    rows, cols = M.shape
    J = np.eye(cols, dtype=dtype)
    tiny = dtype(TINY[dtype]) * np.sum(M * M, dtype=dtype)
    if cols < 2:
        return M, J, 0
    jt2 = dtype(JTOL[dtype]) ** 2
    n = cols + (cols & 1)
    sweeps = 0
    for _ in range(SWEEPS):
        nrm = np.sum(M * M, axis=0, dtype=dtype)
        if all_pairs_test:
            G = M.T @ M
            live = nrm > tiny
            mask = np.triu(np.outer(live, live), 1)
            c = G[mask]
            ab = np.outer(nrm, nrm)[mask]
            if not np.any((c != 0) & (c * c > jt2 * ab)):
                break
        sweeps += 1
        rotated = False
        for step in range(n - 1):
            for k in range(n // 2):
                p, q = rr_pos(k, step, n), rr_pos(n - 1 - k, step, n)
                if p >= cols or q >= cols:
                    continue
                if p > q:
                    p, q = q, p
                c = dtype(M[:, p] @ M[:, q])
                a, b = nrm[p], nrm[q]
                if c != 0 and a > tiny and b > tiny and c * c > jt2 * (a * b):
                    d = b - a
                    t = dtype(math.copysign(2.0 * abs(c), d * c)
                              / (abs(d) + math.sqrt(d * d + 4.0 * c * c)))
                    cs = dtype(1.0 / math.sqrt(t * t + 1.0))
                    sn = cs * t
                    x, y = M[:, p].copy(), M[:, q].copy()
                    M[:, p] = cs * x - sn * y
                    M[:, q] = sn * x + cs * y
                    x, y = J[:, p].copy(), J[:, q].copy()
                    J[:, p] = cs * x - sn * y
                    J[:, q] = sn * x + cs * y
                    nrm[p] = a - t * c
                    nrm[q] = b + t * c
                    rotated = True
        if not rotated:
            break
    return M, J, sweeps


def column_order(M: np.ndarray) -> np.ndarray:
    """Column indices by decreasing squared norm, ties by index
    (cta_order_columns)."""
    s = np.sum(M * M, axis=0)
    return np.array(sorted(range(M.shape[1]), key=lambda j: (-s[j], j)), dtype=np.int64)


def kept(sq_norms_sorted: np.ndarray, rout: int, tol: float) -> int:
    """Columns kept: at most rout and the core's size; with tol > 0 the
    SVDTrunc rule on the squared singular values (at least sigma_0; only
    sigma_0 when sigma_0 < tol^2; else every sigma > tol sigma_0)."""
    keep = min(rout, sq_norms_sorted.size)
    if tol > 0.0 and keep > 0:
        s0, t2 = float(sq_norms_sorted[0]), tol * tol
        c = 1
        if s0 >= t2 * t2:
            while c < keep and float(sq_norms_sorted[c]) > t2 * s0:
                c += 1
        keep = c
    return keep


def round_factors(U: np.ndarray, V: np.ndarray, rout: int, tol: float = 0.0,
                  dtype=np.float64, precondition: bool = False):
    """The general rounding: U V^T (m x n, k terms) to at most rout terms.

    QR of U and of V, core M = R_u R_v^T (min(m, k) x min(n, k)), its Jacobi
    SVD, columns by decreasing norm, the kept count, then
    U_out = Q_u M_out[:, kept], V_out = Q_v J[:, kept] (so U_out has the
    singular values in its column norms and V_out orthonormal columns).

    With `precondition` the Jacobi runs on R_4^T, where M^T = Q_4 R_4 (one
    more QR of the core; Drmac and Veselic, SIAM J. Matrix Anal. Appl. 29,
    2008): R_4^T J = W gives M = W (Q_4 J)^T, so U_out = Q_u W[:, kept] and
    V_out = Q_v Q_4 J[:, kept] keep the same convention, in fewer sweeps on
    graded cores.  A block no taller than its stack (m <= k) skips the QR of
    U: the core is U R_v^T = Q_u M, whose columns have M's inner products, so
    the Jacobi rotations and the rounding are the same, and the rotated
    columns are U_out directly.  Returns (U_out, V_out, sweeps)."""
    U = np.asarray(U, dtype=dtype)
    m, k = U.shape
    Qv, Rv = sla.qr(np.asarray(V, dtype=dtype), mode="economic")
    if m <= k:
        Qu = np.eye(m, dtype=dtype)
        core = U @ Rv.T
    else:
        Qu, Ru = sla.qr(U, mode="economic")
        core = Ru @ Rv.T
    if precondition:
        Q4, R4 = sla.qr(core.T, mode="economic")
        M, J, sweeps = jacobi(R4.T, dtype)
        J = Q4 @ J
    else:
        M, J, sweeps = jacobi(core, dtype)
    order = column_order(M)
    sq = np.sum(M * M, axis=0)[order]
    keep = kept(sq, rout, tol)
    return Qu @ M[:, order[:keep]], Qv @ J[:, order[:keep]], sweeps
