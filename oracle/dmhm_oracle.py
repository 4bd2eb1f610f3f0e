"""CPU oracle: a numpy restatement of the reference's serial H-matrix path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product (``dmhm_b200``) imports
this module; only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s
CPU-baseline leg use it, and only as the checker.

It restates, function by function, the reference's serial ``HMat2d`` /
``HMat3d`` algorithms (YingzhouLi/dmhm v0.2) for real double precision:

* the 64-bit LCG, uniform and Box-Muller Gaussian generators, including the
  width/height quirk of the real ``Dense`` fill,
* the quadtree / octree block structure and natural-to-hierarchical map,
* sparse import, ``SetToRandom``,
* ``Multiply`` / ``TransposeMultiply`` against vectors and dense matrices,
* the H*H ``Multiply`` with randomized low-rank compression, ``RoundedUpdate``,
  ``Compress`` and the dense/low-rank leaf products,
* ``EstimateTwoNorm`` and ``SchulzInvert``,
* ``SetToIdentity`` and ``DirectInvert`` (recursive Schur complements with
  LU-inverted dense leaves).

Each function cites the reference file:line it follows.  The oracle is pinned
against the reference itself: ``oracle/Makefile`` compiles the unmodified
reference sources into ``oracle/_ref/dmhm_ref_driver`` and the fixtures in
``tests/golden/`` (made by ``tests/golden/make_golden.py``) hold its outputs;
``tests/test_oracle_pinned.py`` checks this module against them.

LAPACK calls go through scipy with the same drivers the reference uses
(pivoted QR ``?geqp3``, unpivoted ``?geqrf``, ``?gesvd``), so results agree
with the reference to rounding.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np
import scipy.linalg as sla

# ---------------------------------------------------------------------------
# Random number generation (src/core/random.cpp:13-119,
# include/dmhm/core/random.hpp:100-510, seeds src/core/global.cpp:86-93)
# ---------------------------------------------------------------------------
MASK64 = (1 << 64) - 1
LCG_MULT = 6364136223846793005   # Knuth, random.cpp:15-16 (16-bit limbs)
LCG_ADD = 1442695040888963407
LCG_SEED = (21 << 32) | 17       # Initialize(): seed.d[0]=17, seed.d[1]=21


def lcg_jump(n: int):
    """Affine map (a^n, c (a^n - 1)/(a - 1)) mod 2^64 advancing the LCG n draws.

    Same role as IntegerPowerWith64BitMod (random.cpp:32-65) used for the
    parallel-stream skip-ahead.
    """
    am, cm = 1, 0
    a, c = LCG_MULT, LCG_ADD
    while n:
        if n & 1:
            am, cm = (a * am) & MASK64, (a * cm + c) & MASK64
        a, c = (a * a) & MASK64, (a * c + c) & MASK64
        n >>= 1
    return am, cm


class Lcg:
    """One LCG stream; ``state`` is the value returned by the next draw.

    SerialLcg / ParallelLcg (random.cpp:103-117): return the state, then
    state := a*state + c mod 2^64.  With one rank the parallel stream has the
    serial coefficients and the same seed (SeedParallelLcg, random.cpp:70-101).
    """

    def __init__(self, state: int = LCG_SEED):
        self.state = state & MASK64

    def states(self, n: int) -> np.ndarray:
        """The next n raw states as uint64 (vectorised), advancing the stream."""
        out = np.empty(n, dtype=np.uint64)
        if n == 0:
            return out
        blk = min(n, 1024)
        s = self.state
        for i in range(blk):
            out[i] = s
            s = (LCG_MULT * s + LCG_ADD) & MASK64
        if n > blk:
            aj, cj = lcg_jump(blk)
            aj, cj = np.uint64(aj), np.uint64(cj)
            with np.errstate(over="ignore"):
                for start in range(blk, n, blk):
                    stop = min(start + blk, n)
                    out[start:stop] = out[start - blk:stop - blk] * aj + cj
        am, cm = lcg_jump(n)
        self.state = (am * self.state + cm) & MASK64
        return out

    def uniforms(self, n: int) -> np.ndarray:
        """SerialUniform<double> (random.hpp:250-258): (upper32 + 1) / 2^32."""
        st = self.states(n)
        return ((st >> np.uint64(32)).astype(np.float64) + 1.0) / 4294967296.0

    def uniform(self) -> float:
        return float(self.uniforms(1)[0])

    # Box-Muller on a pair of uniforms (random.hpp:280-292); libm-exact via math.
    @staticmethod
    def _pairs(u: np.ndarray):
        U, V = u[0::2], u[1::2]
        A = np.array([math.sqrt(-2.0 * math.log(x)) for x in U])
        ang = [2.0 * math.pi * v for v in V]
        c = np.array([math.cos(t) for t in ang])
        s = np.array([math.sin(t) for t in ang])
        return A * c, A * s

    def gaussian_vector(self, n: int) -> np.ndarray:
        """SerialGaussianRandomVector (random.hpp:344-364)."""
        x = np.zeros(n)
        if n == 0:
            return x
        pairs = (n + 1) // 2
        X, Y = self._pairs(self.uniforms(2 * pairs))
        x[0:2 * (pairs - 1):2] = X[:pairs - 1]
        x[1:2 * (pairs - 1):2] = Y[:pairs - 1]
        if n & 1:
            x[n - 1] = X[pairs - 1]
        else:
            x[n - 2] = X[pairs - 1]
            x[n - 1] = Y[pairs - 1]
        return x

    def gaussian_vectors(self, m: int, n: int, prev=None) -> np.ndarray:
        """SerialGaussianRandomVectors(Dense<Real>) (random.hpp:418-445).

        Quirk kept: the tail of each column is written at rows n-2, n-1 (the
        WIDTH) rather than m-2, m-1, so rows m-2, m-1 are not written and keep
        what the buffer held: ``prev`` is the old column-major buffer contents
        (Dense::Resize keeps the std::vector, dense.hpp:254-282; new entries
        are zero).  Writes past the column (n > m) would spill into the next
        column; that case is rejected.
        """
        flat = np.zeros(m * n)
        if prev is not None:
            pv = np.asarray(prev, dtype=np.float64).ravel(order="F")[:m * n]
            flat[:pv.size] = pv
        A = flat.reshape((m, n), order="F")
        if m == 0 or n == 0:
            return A
        if n > m:
            raise ValueError("Gaussian fill with width > height spills columns")
        pairs = (m + 1) // 2
        X, Y = self._pairs(self.uniforms(2 * pairs * n))
        X = X.reshape(n, pairs)
        Y = Y.reshape(n, pairs)
        for j in range(n):
            col = A[:, j]
            col[0:2 * (pairs - 1):2] = X[j, :pairs - 1]
            col[1:2 * (pairs - 1):2] = Y[j, :pairs - 1]
            if m & 1:
                col[n - 1] = X[j, pairs - 1]
            else:
                col[n - 2] = X[j, pairs - 1]
                col[n - 1] = Y[j, pairs - 1]
        return A


class Rng:
    """The two global streams of Initialize (global.cpp:86-93)."""

    def __init__(self, oversample: int = 4):
        self.serial = Lcg(LCG_SEED)
        self.parallel = Lcg(LCG_SEED)
        self.oversample = oversample   # Oversample() (global.cpp:30, :155-159)


# ---------------------------------------------------------------------------
# Tree structure (hmat2d.hpp:288-356, HMat2d.cpp:27-87, 797-809;
# 3-D hmat3d.hpp:455-535, HMat3d.cpp:29-110, 852-875)
# ---------------------------------------------------------------------------
def natural_to_hierarchical_map(sizes, num_levels: int) -> np.ndarray:
    """BuildNaturalToHierarchicalMap (HMat2d.cpp:27-87; 3-D HMat3d.cpp:29-110).

    ``sizes`` is (x, y) or (x, y, z); returns map[natural index] = hierarchical
    index with natural order x fastest.
    """
    d = len(sizes)
    total = int(np.prod(sizes))
    mp = np.full(total, -1, dtype=np.int64)
    strides = [1, sizes[0], sizes[0] * sizes[1]][:d]
    counter = [0]

    def rec(origin, this, level):
        if level == num_levels - 1:
            if d == 2:
                for j in range(this[1]):
                    for i in range(this[0]):
                        mp[(origin[1] + j) * strides[1] + origin[0] + i] = counter[0]
                        counter[0] += 1
            else:
                for k in range(this[2]):
                    for j in range(this[1]):
                        for i in range(this[0]):
                            mp[(origin[2] + k) * strides[2] + (origin[1] + j) * strides[1]
                               + origin[0] + i] = counter[0]
                            counter[0] += 1
            return
        lo = [s // 2 for s in this]
        hi = [s - l for s, l in zip(this, lo)]
        for q in range(1 << d):
            bits = [(q >> b) & 1 for b in range(d)]
            sub = [hi[b] if bits[b] else lo[b] for b in range(d)]
            org = [origin[b] + (lo[b] if bits[b] else 0) for b in range(d)]
            rec(org, sub, level + 1)

    rec([0] * d, list(sizes), 0)
    assert counter[0] == total
    return mp


def stencil_csr(sizes, coef: np.ndarray, num_levels: int, shift: float = 0.1):
    """The grid operator of the workloads in hierarchical order, as CSR.

    5-point (2-D) / 7-point (3-D) stencil, diagonal 2*d*c_i + shift, off
    diagonals -min(c_i, c_j); rows built like tests/HMat2d/Invert.cpp:140-181
    (neighbour order x-1, x+1, y-1, y+1[, z-1, z+1], then the diagonal).
    Returns (row_offsets, col_indices, values, map).
    """
    d = len(sizes)
    nx = sizes[0]
    ny = sizes[1]
    N = int(np.prod(sizes))
    mp = natural_to_hierarchical_map(sizes, num_levels)
    inv = np.empty(N, dtype=np.int64)
    inv[mp] = np.arange(N)
    rows, cols, vals = [0], [], []
    for i in range(N):
        nat = int(inv[i])
        x = nat % nx
        y = (nat // nx) % ny
        z = nat // (nx * ny)
        ci = coef[nat]
        nb = []
        if x > 0:
            nb.append(nat - 1)
        if x < nx - 1:
            nb.append(nat + 1)
        if y > 0:
            nb.append(nat - nx)
        if y < ny - 1:
            nb.append(nat + nx)
        if d == 3:
            nz = sizes[2]
            if z > 0:
                nb.append(nat - nx * ny)
            if z < nz - 1:
                nb.append(nat + nx * ny)
        for j in nb:
            cols.append(int(mp[j]))
            vals.append(-min(ci, coef[j]))
        cols.append(int(mp[nat]))
        vals.append(2.0 * d * ci + shift)
        rows.append(len(cols))
    return (np.array(rows, dtype=np.int64), np.array(cols, dtype=np.int64),
            np.array(vals, dtype=np.float64), mp)


NODE, LOW_RANK, DENSE = "node", "low_rank", "dense"


@dataclass
class HMat:
    """One H-matrix block (the Block union of hmat2d.hpp:319-356), real double.

    ``children`` are indexed s + 2^d * t (hmat2d.hpp:288-303 ``Child``);
    low-rank blocks store A = U V^T (low_rank.hpp:22-38).
    """
    dim: int
    num_levels: int
    max_rank: int
    strong: bool
    src_sizes: tuple
    tgt_sizes: tuple
    src_coords: tuple
    tgt_coords: tuple
    src_off: int = 0
    tgt_off: int = 0
    kind: str = NODE
    children: List["HMat"] = field(default_factory=list)
    U: Optional[np.ndarray] = None
    V: Optional[np.ndarray] = None
    D: Optional[np.ndarray] = None

    # -- geometry -----------------------------------------------------------
    @property
    def height(self) -> int:
        return int(np.prod(self.tgt_sizes))

    @property
    def width(self) -> int:
        return int(np.prod(self.src_sizes))

    @property
    def nchild_side(self) -> int:
        return 1 << self.dim

    def admissible(self) -> bool:
        """Admissible (HMat2d.cpp:797-809, HMat3d.cpp:852-875)."""
        dif = [abs(s - t) for s, t in zip(self.src_coords, self.tgt_coords)]
        if self.strong:
            return max(dif) > 1
        return any(v != 0 for v in dif)

    def child_geometry(self):
        """Node ctor (hmat2d.hpp:362-389): half sizes, 2x+bit coordinates."""
        d = self.dim
        lo_s = [s // 2 for s in self.src_sizes]
        hi_s = [s - l for s, l in zip(self.src_sizes, lo_s)]
        lo_t = [s // 2 for s in self.tgt_sizes]
        hi_t = [s - l for s, l in zip(self.tgt_sizes, lo_t)]
        q = self.nchild_side

        def sub(lo, hi, idx):
            return tuple(hi[b] if (idx >> b) & 1 else lo[b] for b in range(d))

        src_sub = [sub(lo_s, hi_s, s) for s in range(q)]
        tgt_sub = [sub(lo_t, hi_t, t) for t in range(q)]
        src_sz = [int(np.prod(x)) for x in src_sub]
        tgt_sz = [int(np.prod(x)) for x in tgt_sub]
        out = []
        toff = self.tgt_off
        for t in range(q):
            soff = self.src_off
            for s in range(q):
                out.append(dict(
                    src_sizes=src_sub[s], tgt_sizes=tgt_sub[t],
                    src_coords=tuple(2 * self.src_coords[b] + ((s >> b) & 1) for b in range(d)),
                    tgt_coords=tuple(2 * self.tgt_coords[b] + ((t >> b) & 1) for b in range(d)),
                    src_off=soff, tgt_off=toff,
                    s_local=soff - self.src_off, t_local=toff - self.tgt_off))
                soff += src_sz[s]
            toff += tgt_sz[t]
        return out

    def new_child(self, g) -> "HMat":
        return HMat(self.dim, self.num_levels - 1, self.max_rank, self.strong,
                    g["src_sizes"], g["tgt_sizes"], g["src_coords"], g["tgt_coords"],
                    g["src_off"], g["tgt_off"])

    def child(self, t: int, s: int) -> "HMat":
        return self.children[s + self.nchild_side * t]

    def child_ranges(self):
        """(t, s, row slice, col slice) relative to this block, in order."""
        for idx, g in enumerate(self.child_geometry()):
            t, s = divmod(idx, self.nchild_side)
            c = self.children[idx]
            yield t, s, slice(g["t_local"], g["t_local"] + c.height), \
                slice(g["s_local"], g["s_local"] + c.width)

    def shell(self) -> "HMat":
        return HMat(self.dim, self.num_levels, self.max_rank, self.strong,
                    self.src_sizes, self.tgt_sizes, self.src_coords, self.tgt_coords,
                    self.src_off, self.tgt_off)

    @property
    def rank(self) -> int:
        return 0 if self.U is None else self.U.shape[1]

    def leaves(self):
        if self.kind == NODE:
            for c in self.children:
                yield from c.leaves()
        else:
            yield self


def top_level(dim, sizes, num_levels, max_rank, strong=True) -> HMat:
    sizes = tuple(sizes)
    zero = tuple([0] * dim)
    return HMat(dim, num_levels, max_rank, strong, sizes, sizes, zero, zero, 0, 0)


def import_sparse(H: HMat, rows, cols, vals) -> HMat:
    """ImportSparse (HMat2d.cpp:961-1033) + ConvertSubmatrix
    (src/hmat_tools/ConvertSubmatrix.cpp:14-119); S.symmetric = false."""
    i0, j0, m, n = H.tgt_off, H.src_off, H.height, H.width
    if H.admissible():
        us, vs = [], []
        for i in range(m):
            for k in range(rows[i0 + i], rows[i0 + i + 1]):
                j = cols[k]
                if j0 <= j < j0 + n:
                    us.append(i)
                    vs.append((j - j0, vals[k]))
        r = len(us)
        H.kind = LOW_RANK
        H.U = np.zeros((m, r))
        H.V = np.zeros((n, r))
        for q in range(r):
            H.U[us[q], q] = 1.0
            H.V[vs[q][0], q] = vs[q][1]
    elif H.num_levels > 1:
        H.kind = NODE
        H.children = [import_sparse(H.new_child(g), rows, cols, vals)
                      for g in H.child_geometry()]
    else:
        H.kind = DENSE
        D = np.zeros((m, n))
        for i in range(m):
            for k in range(rows[i0 + i], rows[i0 + i + 1]):
                j = cols[k]
                if j0 <= j < j0 + n:
                    D[i, j - j0] = vals[k]
        H.D = D
    return H


def set_to_random(H: HMat, rng: Rng):
    """SetToRandom (src/HMat2d/SetToRandom-incl.hpp:14-55): parallel stream,
    dense leaves refilled in place, low-rank blocks resized to rank max_rank
    (U then V); entries the fill skips keep the old buffer contents."""
    if H.kind == NODE:
        for c in H.children:
            set_to_random(c, rng)
    elif H.kind == DENSE:
        H.D = rng.parallel.gaussian_vectors(H.height, H.width, prev=H.D)
    else:
        H.U = rng.parallel.gaussian_vectors(H.height, H.max_rank, prev=H.U)
        H.V = rng.parallel.gaussian_vectors(H.width, H.max_rank, prev=H.V)


# ---------------------------------------------------------------------------
# H-matrix times dense (src/HMat2d/MultiplyDense-incl.hpp:12-232,
# leaf products src/hmat_tools/MultiplyMatrix.cpp:31-199 and the
# TransposeMultiplyMatrix.cpp counterparts)
# ---------------------------------------------------------------------------
def multiply_dense(H: HMat, alpha: float, B: np.ndarray, beta: float = 0.0,
                   C: Optional[np.ndarray] = None) -> np.ndarray:
    """C := alpha H B + beta C."""
    B = np.asarray(B, dtype=np.float64)
    if B.ndim == 1:
        return multiply_dense(H, alpha, B[:, None], beta,
                              None if C is None else C[:, None])[:, 0]
    if C is None:
        C = np.zeros((H.height, B.shape[1]))
    else:
        C = C * beta if beta != 1.0 else C.copy()
    _mul_acc(H, alpha, B, C, transpose=False)
    return C


def transpose_multiply_dense(H: HMat, alpha: float, B: np.ndarray) -> np.ndarray:
    """C := alpha H^T B (MultiplyDense-incl.hpp:70-150)."""
    B = np.asarray(B, dtype=np.float64)
    if B.ndim == 1:
        return transpose_multiply_dense(H, alpha, B[:, None])[:, 0]
    C = np.zeros((H.width, B.shape[1]))
    _mul_acc(H, alpha, B, C, transpose=True)
    return C


def _mul_acc(H: HMat, alpha, B, C, transpose: bool):
    if H.kind == NODE:
        for t, s, rs, cs in H.child_ranges():
            if transpose:
                _mul_acc(H.child(t, s), alpha, B[rs], C[cs], True)
            else:
                _mul_acc(H.child(t, s), alpha, B[cs], C[rs], False)
    elif H.kind == LOW_RANK:
        if H.rank == 0:
            return
        if transpose:   # C += alpha V (U^T B)
            C += alpha * (H.V @ (H.U.T @ B))
        else:           # C += alpha U (V^T B)   MultiplyMatrix.cpp:144-199
            C += alpha * (H.U @ (H.V.T @ B))
    else:
        C += alpha * ((H.D.T if transpose else H.D) @ B)


# ---------------------------------------------------------------------------
# Leaf algebra (src/hmat_tools/*.cpp)
# ---------------------------------------------------------------------------
@dataclass
class LR:
    U: np.ndarray
    V: np.ndarray

    @property
    def rank(self):
        return self.U.shape[1]


def lr_times_lr(alpha, A: LR, B: LR) -> LR:
    """F := alpha F F (MultiplyMatrix.cpp:245-312)."""
    if A.rank <= B.rank:
        W = B.U.T @ A.V
        return LR(A.U.copy(), alpha * (B.V @ W))
    W = A.V.T @ B.U
    return LR(alpha * (A.U @ W), B.V.copy())


# CompressionTolerance (src/core/global.cpp:160-181): 0 keeps the fixed rank
# of HMat2d; > 0 truncates every SVD as the single-rank DistHMat does
# (SVDTrunc, src/DistHMat2d/Truncation-incl.hpp:37-63): keep the singular
# values above tol * sigma_0 (at least sigma_0; only sigma_0 when sigma_0 <
# tol^2, the cutoff index 0 of Truncation-incl.hpp:52-55), at most the rank cap.
_COMPRESSION_TOL = [0.0]


def set_compression_tolerance(tol: float):
    _COMPRESSION_TOL[0] = float(tol)


def _kept(s: np.ndarray, cap: int) -> int:
    tol = _COMPRESSION_TOL[0]
    if tol <= 0.0:
        return cap
    if s.size == 0 or cap == 0:
        return 0
    if s[0] < tol * tol:
        return 1
    return int(min(cap, max(1, np.count_nonzero(s > tol * s[0]))))


def rounded_update(max_rank: int, alpha, A: LR, beta, B: LR) -> LR:
    """B :~= alpha A + beta B (src/hmat_tools/RoundedUpdate.cpp:14-162)."""
    m, n = A.U.shape[0], A.V.shape[0]
    min_dim = min(m, n)
    r = A.rank + B.rank
    rr = min(r, min_dim, max_rank)
    if rr == r:   # exact concatenation, :35-53
        return LR(np.hstack([beta * B.U, alpha * A.U]), np.hstack([B.V, A.V]))
    U = np.hstack([alpha * A.U, beta * B.U])
    V = np.hstack([A.V, B.V])
    QU, RU = sla.qr(U, mode="economic")
    QV, RV = sla.qr(V, mode="economic")
    W = RU @ RV.T
    Uw, s, VTw = sla.svd(W, full_matrices=False, lapack_driver="gesvd")
    rr = _kept(s, rr)
    return LR(QU @ (Uw[:, :rr] * s[:rr]), QV @ VTw[:rr].T)


def compress_dense(max_rank: int, D: np.ndarray) -> LR:
    """Compress(maxRank, D, F) (src/hmat_tools/Compress.cpp:14-53) and the
    D*D->F path (MultiplyMatrix.cpp:405-449): SVD, keep min(minDim, maxRank)."""
    m, n = D.shape
    r = min(m, n, max_rank)
    U, s, VT = sla.svd(D, full_matrices=False, lapack_driver="gesvd")
    r = _kept(s, r)
    return LR(U[:, :r].copy(), VT[:r].T * s[:r])


def randomized_product(sample_rank: int, alpha, A: HMat, B: HMat, rng: Rng) -> LR:
    """F := alpha A B by randomized sampling (include/dmhm/hmat_tools.hpp:1657-1746)."""
    r = min(A.max_rank, B.max_rank, min(A.height, A.width), min(B.height, B.width))
    Omega = rng.serial.gaussian_vectors(B.width, sample_rank)
    X = multiply_dense(B, alpha, Omega)
    Y = multiply_dense(A, 1.0, X)
    Q, _, _ = sla.qr(Y, mode="economic", pivoting=True)     # geqp3 + orgqr
    X = transpose_multiply_dense(A, alpha, Q)
    FV = transpose_multiply_dense(B, 1.0, X)
    Us, s, VT = sla.svd(FV, full_matrices=False, lapack_driver="gesvd")
    r = _kept(s, min(r, s.size))
    V = Us[:, :r].copy()
    U = Q @ (VT[:r].T * s[:r])
    return LR(U, V)


def randomized_transpose_product(sample_rank: int, alpha, A: HMat, B: HMat, rng: Rng) -> LR:
    """F := alpha A^T B by randomized sampling (TransposeMultiply,
    include/dmhm/hmat_tools.hpp:1848-1937; AdjointMultiply, :2039-, is the
    same for real scalars): Y = A^T (alpha B Omega), Q = orth(Y),
    F.V = B^T (alpha A Q), truncated SVD, F.U = Q (Sigma V^T)^T."""
    r = min(A.max_rank, B.max_rank, min(A.height, A.width), min(B.height, B.width))
    Omega = rng.serial.gaussian_vectors(B.width, sample_rank)
    X = multiply_dense(B, alpha, Omega)
    Y = transpose_multiply_dense(A, 1.0, X)
    Q, _, _ = sla.qr(Y, mode="economic", pivoting=True)     # geqp3 + orgqr
    X = multiply_dense(A, alpha, Q)
    FV = transpose_multiply_dense(B, 1.0, X)
    Us, s, VT = sla.svd(FV, full_matrices=False, lapack_driver="gesvd")
    r = _kept(s, min(r, s.size))
    V = Us[:, :r].copy()
    U = Q @ (VT[:r].T * s[:r])
    return LR(U, V)


def _low_rank_of(H: HMat) -> LR:
    return LR(H.U, H.V)


def _product_low_rank(alpha, A: HMat, B: HMat, C: HMat, rng: Rng):
    """The low-rank W := alpha A B of the admissible-C cases
    (MultiplyHMat-incl.hpp:45-95 and :206-266); returns LR, or a dense
    matrix for the dense-dense case (compressed by the caller)."""
    if A.kind == LOW_RANK and B.kind == LOW_RANK:
        return lr_times_lr(alpha, _low_rank_of(A), _low_rank_of(B))
    if A.kind == LOW_RANK and B.kind == NODE:
        return LR(A.U.copy(), transpose_multiply_dense(B, alpha, A.V))
    if A.kind == LOW_RANK and B.kind == DENSE:
        return LR(A.U.copy(), alpha * (B.D.T @ A.V))
    if A.kind == NODE and B.kind == LOW_RANK:
        return LR(multiply_dense(A, alpha, B.U), B.V.copy())
    if A.kind == NODE and B.kind == NODE:
        return randomized_product(C.max_rank + rng.oversample, alpha, A, B, rng)
    if A.kind == DENSE and B.kind == LOW_RANK:
        return LR(alpha * (A.D @ B.U), B.V.copy())
    if A.kind == DENSE and B.kind == DENSE:
        return alpha * (A.D @ B.D)
    raise ValueError("invalid H-matrix combination")


def import_low_rank(C: HMat, F: LR):
    """ImportLowRank (HMat2d.cpp:811-904)."""
    C.children, C.U, C.V, C.D = [], None, None, None
    if C.admissible():
        C.kind = LOW_RANK
        C.U, C.V = F.U.copy(), F.V.copy()
    elif C.num_levels > 1:
        C.kind = NODE
        geo = C.child_geometry()
        for g in geo:
            ch = C.new_child(g)
            sub = LR(F.U[g["t_local"]:g["t_local"] + ch.height],
                     F.V[g["s_local"]:g["s_local"] + ch.width])
            import_low_rank(ch, sub)
            C.children.append(ch)
    else:
        C.kind = DENSE
        C.D = F.U @ F.V.T


def update_with_low_rank(C: HMat, alpha, F: LR):
    """UpdateWithLowRank (HMat2d.cpp:906-959)."""
    if C.admissible():
        nf = rounded_update(C.max_rank, alpha, F, 1.0, _low_rank_of(C))
        C.U, C.V = nf.U, nf.V
    elif C.num_levels > 1:
        for t, s, rs, cs in C.child_ranges():
            update_with_low_rank(C.child(t, s), alpha, LR(F.U[rs], F.V[cs]))
    else:
        C.D = C.D + alpha * (F.U @ F.V.T)


def scale(H: HMat, alpha):
    """Scale (HMat2d.cpp:616-647, hmat_tools.hpp Scale(LowRank): alpha=0 drops rank)."""
    if H.kind == NODE:
        for c in H.children:
            scale(c, alpha)
    elif H.kind == LOW_RANK:
        if alpha == 0:
            H.U = np.zeros((H.height, 0))
            H.V = np.zeros((H.width, 0))
        else:
            H.U = alpha * H.U
    else:
        H.D = alpha * H.D


def hh_multiply(A: HMat, alpha, B: HMat, rng: Rng) -> HMat:
    """C := alpha A B (src/HMat2d/MultiplyHMat-incl.hpp:12-187)."""
    C = HMat(A.dim, A.num_levels, A.max_rank, A.strong or B.strong,
             B.src_sizes, A.tgt_sizes, B.src_coords, A.tgt_coords,
             B.src_off, A.tgt_off)
    if C.admissible():
        C.kind = LOW_RANK
        W = _product_low_rank(alpha, A, B, C, rng)
        if isinstance(W, np.ndarray):
            W = compress_dense(C.max_rank, W)
        C.U, C.V = W.U, W.V
    elif C.num_levels > 1:
        C.kind = NODE
        if A.kind == DENSE or B.kind == DENSE:
            raise ValueError("invalid H-matrix combination")
        if A.kind == LOW_RANK or B.kind == LOW_RANK:
            import_low_rank(C, _product_low_rank(alpha, A, B, C, rng))
        else:
            q = A.nchild_side
            kids = [None] * (q * q)
            for t in range(q):
                for s in range(q):
                    ch = hh_multiply(A.child(t, 0), alpha, B.child(0, s), rng)
                    for u in range(1, q):
                        hh_multiply_update(A.child(t, u), alpha, B.child(u, s), 1.0, ch, rng)
                    kids[s + q * t] = ch
            C.children = kids
    else:
        C.kind = DENSE
        if A.kind == NODE or B.kind == NODE:
            raise ValueError("invalid H-matrix combination")
        Ad = A.D if A.kind == DENSE else A.U @ A.V.T
        if A.kind == LOW_RANK and B.kind == LOW_RANK:
            W = lr_times_lr(alpha, _low_rank_of(A), _low_rank_of(B))
            C.D = W.U @ W.V.T
        elif A.kind == LOW_RANK:
            C.D = alpha * (A.U @ (A.V.T @ B.D))
        elif B.kind == LOW_RANK:
            C.D = alpha * ((Ad @ B.U) @ B.V.T)
        else:
            C.D = alpha * (A.D @ B.D)
    return C


def hh_multiply_update(A: HMat, alpha, B: HMat, beta, C: HMat, rng: Rng):
    """C :~= alpha A B + beta C (src/HMat2d/MultiplyHMat-incl.hpp:189-380)."""
    if C.admissible():
        if A.kind == DENSE and B.kind == DENSE:
            D = alpha * (A.D @ B.D)
            if C.rank:
                D = D + beta * (C.U @ C.V.T)
            W = compress_dense(C.max_rank, D)
            C.U, C.V = W.U, W.V
            return
        W = _product_low_rank(alpha, A, B, C, rng)
        nf = rounded_update(C.max_rank, 1.0, W, beta, _low_rank_of(C))
        C.U, C.V = nf.U, nf.V
    elif C.num_levels > 1:
        if A.kind == LOW_RANK or B.kind == LOW_RANK:
            W = _product_low_rank(alpha, A, B, C, rng)
            scale(C, beta)
            update_with_low_rank(C, 1.0, W)
        else:
            q = A.nchild_side
            for t in range(q):
                for s in range(q):
                    hh_multiply_update(A.child(t, 0), alpha, B.child(0, s), beta,
                                       C.child(t, s), rng)
                    for u in range(1, q):
                        hh_multiply_update(A.child(t, u), alpha, B.child(u, s), 1.0,
                                           C.child(t, s), rng)
    else:
        if A.kind == LOW_RANK and B.kind == LOW_RANK:
            W = lr_times_lr(alpha, _low_rank_of(A), _low_rank_of(B))
            P = W.U @ W.V.T
        elif A.kind == LOW_RANK:
            P = alpha * (A.U @ (A.V.T @ B.D))
        elif B.kind == LOW_RANK:
            P = alpha * ((A.D @ B.U) @ B.V.T)
        else:
            P = alpha * (A.D @ B.D)
        C.D = beta * C.D + P


def copy(H: HMat) -> HMat:
    """CopyFrom (HMat2d.cpp:331-391)."""
    C = H.shell()
    C.kind = H.kind
    if H.kind == NODE:
        C.children = [copy(c) for c in H.children]
    elif H.kind == LOW_RANK:
        C.U, C.V = H.U.copy(), H.V.copy()
    else:
        C.D = H.D.copy()
    return C


def adjoint(H: HMat) -> HMat:
    """AdjointFrom (HMat2d.cpp:545-614): real case = transpose."""
    C = HMat(H.dim, H.num_levels, H.max_rank, H.strong,
             H.tgt_sizes, H.src_sizes, H.tgt_coords, H.src_coords,
             H.tgt_off, H.src_off)
    C.kind = H.kind
    if H.kind == NODE:
        q = H.nchild_side
        C.children = [None] * (q * q)
        for t in range(q):
            for s in range(q):
                C.children[s + q * t] = adjoint(H.child(s, t))
    elif H.kind == LOW_RANK:
        C.U, C.V = H.V.copy(), H.U.copy()
    else:
        C.D = H.D.T.copy()
    return C


def add_constant_to_diagonal(H: HMat, alpha):
    """AddConstantToDiagonal (HMat2d.cpp:704-744)."""
    if H.kind == NODE:
        for i in range(H.nchild_side):
            add_constant_to_diagonal(H.child(i, i), alpha)
    elif H.kind == DENSE:
        k = min(H.D.shape)
        H.D[np.arange(k), np.arange(k)] += alpha


def set_to_identity(H: HMat):
    """SetToIdentity (src/HMat2d/HMat2d.cpp:650-702): diagonal children
    recursively, Scale(0) elsewhere (low-rank blocks drop to rank 0); a dense
    block becomes the leading identity.  A low-rank block is left alone, as
    the RELEASE build does."""
    if H.kind == NODE:
        q = H.nchild_side
        for t in range(q):
            for s in range(q):
                if s == t:
                    set_to_identity(H.child(t, s))
                else:
                    scale(H.child(t, s), 0.0)
    elif H.kind == DENSE:
        H.D = np.zeros_like(H.D)
        k = min(H.D.shape)
        H.D[np.arange(k), np.arange(k)] = 1.0


def invert_dense(D: np.ndarray) -> np.ndarray:
    """hmat_tools::Invert, non-symmetric branch (src/hmat_tools/Invert.cpp
    :14-42): LU with partial pivoting (?getrf) and the inverse from the
    factors (?getri, workspace n * 32 as lapack.hpp:1500-1504)."""
    from scipy.linalg import lapack
    n = D.shape[0]
    lu, piv, info = lapack.dgetrf(np.asfortranarray(D))
    if info < 0:
        raise ValueError("dgetrf: bad argument %d" % -info)
    inv, info = lapack.dgetri(lu, piv, lwork=max(1, 32 * n))
    if info < 0:
        raise ValueError("dgetri: bad argument %d" % -info)
    return np.array(inv)


def direct_invert(H: HMat, rng: Rng):
    """A := inv(A) in place by recursive Schur complements (DirectInvert,
    src/HMat2d/Invert-incl.hpp:17-125; 3-D src/HMat3d/Invert-incl.hpp:14-122).

    Block Gauss-Jordan over the 2^d x 2^d children: B keeps a copy of A, A
    starts as the identity; for each pivot l the diagonal child is inverted
    recursively, row l of A and of B is multiplied by it, and the rows below
    are eliminated; a backward sweep then clears the rows above.  Every
    product is the H*H product above (fresh for the row scalings, the
    update form for the eliminations), in the reference's order, so the
    generator is drawn in the same sequence."""
    if H.kind == DENSE:
        H.D = invert_dense(H.D)
        return
    if H.kind != NODE:
        return
    q = H.nchild_side
    B = copy(H)
    set_to_identity(H)
    A = H

    def put(M: HMat, t: int, s: int, X: HMat):
        M.children[s + q * t] = X

    for l in range(q):
        put(A, l, l, copy(B.child(l, l)))
        direct_invert(A.child(l, l), rng)
        for j in range(l):
            C = copy(A.child(l, j))
            put(A, l, j, hh_multiply(A.child(l, l), 1.0, C, rng))
        for j in range(l + 1, q):
            C = copy(B.child(l, j))
            put(B, l, j, hh_multiply(A.child(l, l), 1.0, C, rng))
        for i in range(l + 1, q):
            for j in range(l + 1):
                hh_multiply_update(B.child(i, l), -1.0, A.child(l, j), 1.0, A.child(i, j), rng)
            for j in range(l + 1, q):
                hh_multiply_update(B.child(i, l), -1.0, B.child(l, j), 1.0, B.child(i, j), rng)
    for l in range(q - 1, -1, -1):
        for i in range(l - 1, -1, -1):
            for j in range(q):
                hh_multiply_update(B.child(i, l), -1.0, A.child(l, j), 1.0, A.child(i, j), rng)


def estimate_two_norm(H: HMat, theta: float, confidence: float, rng: Rng) -> float:
    """EstimateTwoNorm (include/dmhm/hmat_tools.hpp:1504-1548)."""
    n = H.height
    k = int(math.ceil(math.log(0.8 * math.sqrt(n) * math.pow(10, confidence)) / math.log(theta)))
    x = rng.serial.gaussian_vector(n)
    x = x * (1.0 / np.sqrt(np.dot(x, x)))
    est = theta
    root = 1.0 / k
    for _ in range(k):
        x = multiply_dense(H, 1.0, x)
        nrm = float(np.sqrt(np.dot(x, x)))
        x = x * (1.0 / nrm)
        est *= math.pow(nrm, root)
    return est


def schulz_invert(A: HMat, num_iterations: int, rng: Rng, theta=1.5,
                  confidence=6.0, stop_tol=1e-4):
    """SchulzInvert (src/HMat2d/Invert-incl.hpp:127-196).

    Returns (X, iterations run, [estimate of ||A||, ||I - X_k A|| per check]).
    """
    stop = False
    if num_iterations <= 0:
        num_iterations = 30
        stop = True
    est = estimate_two_norm(A, theta, confidence, rng)
    trace = [est]
    alpha = 2.0 / (est * est)
    X = adjoint(A)
    scale(X, alpha)
    k = 0
    while k < num_iterations:
        Z = hh_multiply(X, -1.0, A, rng)
        if stop:
            add_constant_to_diagonal(Z, 1.0)
            ez = estimate_two_norm(Z, theta, confidence, rng)
            trace.append(ez)
            if abs(ez) < stop_tol:
                add_constant_to_diagonal(Z, 1.0)
                X = hh_multiply(Z, 1.0, X, rng)
                k += 1
                break
            add_constant_to_diagonal(Z, 1.0)
        else:
            add_constant_to_diagonal(Z, 2.0)
        X = hh_multiply(Z, 1.0, X, rng)
        k += 1
    return X, k, trace


def to_dense(H: HMat) -> np.ndarray:
    return multiply_dense(H, 1.0, np.eye(H.width))


def build_stencil_hmat(dim, sizes, num_levels, max_rank, coef, shift=0.1, strong=True):
    rows, cols, vals, _ = stencil_csr(sizes, coef, num_levels, shift)
    H = top_level(dim, sizes, num_levels, max_rank, strong)
    return import_sparse(H, rows, cols, vals)

