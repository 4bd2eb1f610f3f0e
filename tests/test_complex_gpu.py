"""Complex-double H-matrices (HMat2d<std::complex<double>>, real form on the
device) against dense complex algebra in numpy on the same operator.

Tolerances: products of a sparse-built matrix are exact up to rounding
(relative 1e-13); the H*H square of a sparse-built matrix has exact-rank
blocks (1e-12); SchulzInvert (stopTol 1e-8, maxRank 12) is compared with the
dense inverse on probe vectors to 1e-7, above the truncation floor that
fixed-rank compression leaves (the reference's own complex run of the first
case lands 3e-9 from the dense inverse), as the reference's Invert test
evaluates its result (tests/HMat2d/Invert.cpp:71-104).
"""
import numpy as np
import pytest

import dmhm_b200 as D
from dmhm_b200 import operators as O
from helpers import relerr

pytestmark = pytest.mark.gpu

CASES = [((32, 32), 3, 6.0), ((24, 20), 3, 3.0), ((48, 48), 4, 8.5)]


def make(sizes, levels, k, rank=12, ctx=None):
    S = O.helmholtz(sizes, k, levels)
    ctx = ctx or D.Context(0)
    H = D.HMat2d(S, levels, rank, True, *sizes, ctx=ctx)
    return ctx, S, H


def cplx(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


@pytest.mark.parametrize("sizes,levels,k", CASES)
def test_complex_products(sizes, levels, k):
    ctx, S, H = make(sizes, levels, k)
    assert H.is_complex and H.Height() == S.height
    A = O.dense_from_sparse(S)
    rng = np.random.default_rng(3)
    X = cplx(rng, S.height, 5)
    Y = cplx(rng, S.height, 5)
    al, be = 0.7 - 0.4j, -0.3 + 1.1j
    assert relerr(H.Multiply(al, X), al * A @ X) < 1e-13
    assert relerr(H.Multiply(al, X, be, Y.copy()), al * A @ X + be * Y) < 1e-13
    assert relerr(H.TransposeMultiply(al, X, be, Y.copy()), al * A.T @ X + be * Y) < 1e-13
    assert relerr(H.AdjointMultiply(al, X, be, Y.copy()), al * A.conj().T @ X + be * Y) < 1e-13
    x = X[:, 0]
    assert relerr(H.Multiply(1.0, x), A @ x) < 1e-13   # real scalars, vector


@pytest.mark.parametrize("sizes,levels,k", CASES[:2])
def test_complex_square(sizes, levels, k):
    ctx, S, H = make(sizes, levels, k)
    A = O.dense_from_sparse(S)
    X = cplx(np.random.default_rng(4), S.height, 3)
    H2 = H.Multiply(1.0, H)
    assert relerr(H2.Multiply(1.0, X), A @ (A @ X)) < 1e-12


@pytest.mark.parametrize("sizes,levels,k", CASES)
def test_complex_schulz(sizes, levels, k):
    ctx, S, H = make(sizes, levels, k)
    A = O.dense_from_sparse(S)
    its, trace = H.SchulzInvert(-1, 1.5, 6.0, 1e-8)
    # maxRank 12 leaves a truncation floor near 1e-8 in the worst direction
    # of ||I - X A|| (the reference's own run of the first case ends within
    # 3e-9 of the dense inverse on probes, as this one must)
    assert trace[-1] < 1e-7 and its <= 30
    # the power-method estimate of ||A|| (first trace entry) bounds the norm
    assert np.linalg.norm(A, 2) <= trace[0] * (1 + 1e-12)
    P = cplx(np.random.default_rng(5), S.height, 4)
    ref = np.linalg.solve(A, P)
    assert relerr(H.Multiply(1.0, P), ref) < 1e-7


def test_complex_mixed_schulz():
    ctx, S, H = make((32, 32), 3, 6.0)
    A = O.dense_from_sparse(S)
    its, low, trace = H.SchulzInvertMixed(-1, 1.5, 6.0, 1e-8, 0.1)
    assert low >= 1 and trace[-1] < 1e-7
    P = cplx(np.random.default_rng(6), S.height, 4)
    assert relerr(H.Multiply(1.0, P), np.linalg.solve(A, P)) < 1e-7


def test_complex_matches_reference():
    """Against the reference's own HMat2d<std::complex<double>> (fixture made
    by tests/golden/make_golden.py): Multiply exactly, A*A exactly (sparse
    factors), SchulzInvert to the truncation level both methods reach (the
    reference's inverse is within 3e-9 of the dense one on these probes)."""
    from helpers import load
    fx = load("cplx")
    sizes = tuple(int(s) for s in fx["sizes"])
    ctx, S, H = make(sizes, int(fx["levels"]), float(fx["kwave"]), rank=int(fx["rank"]))
    ctx.set_oversample(int(fx["oversample"]))
    P = fx["probes"]
    assert relerr(H.Multiply(1.0, P), fx["matvec"]) < 1e-13
    assert relerr(H.Multiply(1.0, H).Multiply(1.0, P), fx["hh_AA"]) < 1e-12
    its, trace = H.SchulzInvert(-1, 1.5, 6.0, 1e-8)
    assert relerr(H.Multiply(1.0, P), fx["schulz_stop"]) < 1e-7


def test_complex_3d_products():
    """HMat3d<std::complex<double>>: seven-point Helmholtz-like operator on an
    8 x 8 x 8 grid, products and the H*H square against dense algebra."""
    sizes = (8, 8, 8)
    S = O.helmholtz(sizes, 4.0, 2)
    ctx = D.Context(0)
    H = D.HMat3d(S, 2, 8, True, *sizes, ctx=ctx)
    assert H.is_complex and H.Height() == 512
    A = O.dense_from_sparse(S)
    X = cplx(np.random.default_rng(7), 512, 3)
    assert relerr(H.Multiply(0.5 + 0.25j, X), (0.5 + 0.25j) * A @ X) < 1e-13
    assert relerr(H.AdjointMultiply(1.0, X), A.conj().T @ X) < 1e-13
    assert relerr(H.Multiply(1.0, H).Multiply(1.0, X), A @ (A @ X)) < 1e-12


def test_complex_scalar_helpers():
    """Scale and AddConstantToDiagonal with complex alpha, ConjugateFrom,
    TransposeFrom (no conjugation) and AdjointFrom, against dense algebra, on
    a weakly admissible matrix built from the operator (its low-rank blocks
    hold the stencil entries between neighbouring boxes exactly)."""
    sizes = (24, 20)
    S = O.helmholtz(sizes, 3.0, 3)
    ctx = D.Context(0)
    H = D.HMat2d(S, 3, 12, False, *sizes, ctx=ctx)
    assert H.BlockCensus()["rank_sum"] > 0
    n = S.height
    A = O.dense_from_sparse(S)
    X = cplx(np.random.default_rng(8), n, 3)
    assert relerr(H.Multiply(1.0, X), A @ X) < 1e-13
    al, be = 0.6 - 1.3j, -0.2 + 0.7j
    H.Scale(al)
    H.AddConstantToDiagonal(be)
    B = al * A + be * np.eye(n)
    assert relerr(H.Multiply(1.0, X), B @ X) < 1e-13
    Hc = D.HMat2d(ctx=ctx).ConjugateFrom(H)
    assert relerr(Hc.Multiply(1.0, X), B.conj() @ X) < 1e-13
    Ht = D.HMat2d(ctx=ctx).TransposeFrom(H)
    assert relerr(Ht.Multiply(1.0, X), B.T @ X) < 1e-13
    Ha = D.HMat2d(ctx=ctx).AdjointFrom(H)
    assert relerr(Ha.Multiply(1.0, X), B.conj().T @ X) < 1e-13
