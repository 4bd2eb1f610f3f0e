"""Tolerance-truncated H*H products (CompressionTolerance, src/core/
global.cpp:160-181, applied as SVDTrunc of src/DistHMat2d/Truncation-incl.hpp
:37-63) on the GPU against the oracle with the same tolerance.

Where the tolerance drops content the GPU and the oracle may take different
(equally accurate) truncation paths, so products are compared at the
tolerance's scale: 1e-7 relative for tol = 1e-10."""
import numpy as np
import pytest

import dmhm_b200 as D
from helpers import build, load, relerr

pytestmark = pytest.mark.gpu


def ctx_for(fx, tol):
    c = D.Context(0)
    c.set_oversample(int(fx["oversample"]))
    c.set_compression_tolerance(tol)
    return c


def test_tolerance_knob_roundtrip():
    c = D.Context(0)
    assert c.compression_tolerance() == 0.0
    c.set_compression_tolerance(1e-9)
    assert c.compression_tolerance() == 1e-9
    with pytest.raises(D.HMError):
        c.set_compression_tolerance(-1.0)


@pytest.mark.parametrize("case", ["c1", "ragged"])
def test_exact_square_keeps_value_and_shrinks_ranks(case):
    """A*A of a sparse-built A is exact: a tiny tolerance must keep the
    product and store it at (much) lower ranks than maxRank."""
    fx = load(case)
    plain = build(D, fx, ctx_for(fx, 0.0))
    Cp = plain.Multiply(1.0, plain)
    c = ctx_for(fx, 1e-12)
    A = build(D, fx, c)
    Ct = A.Multiply(1.0, A)
    assert relerr(Ct.Multiply(1.0, fx["probes"]), fx["hh_AA"]) < 1e-11
    assert Ct.BlockCensus()["rank_sum"] < Cp.BlockCensus()["rank_sum"]


@pytest.mark.parametrize("case", ["c1", "ragged"])
def test_random_factors_against_oracle(case):
    from oracle import dmhm_oracle as O
    fx = load(case)
    tol = 1e-10
    sizes = tuple(int(s) for s in fx["sizes"])
    L, r = int(fx["levels"]), int(fx["rank"])
    c = ctx_for(fx, tol)
    A = build(D, fx, c)
    A.SetToRandom()
    B = build(D, fx, c, "coefB")
    B.SetToRandom()
    Cm = A.Multiply(0.25, B)
    rng = O.Rng(int(fx["oversample"]))
    Ao = O.build_stencil_hmat(2, sizes, L, r, fx["coef"], strong=bool(fx["strong"]))
    O.set_to_random(Ao, rng)
    Bo = O.build_stencil_hmat(2, sizes, L, r, fx["coefB"], strong=bool(fx["strong"]))
    O.set_to_random(Bo, rng)
    O.set_compression_tolerance(tol)
    try:
        Co = O.hh_multiply(Ao, 0.25, Bo, rng)
    finally:
        O.set_compression_tolerance(0.0)
    P = fx["probes"]
    assert relerr(Cm.Multiply(1.0, P), O.multiply_dense(Co, 1.0, P)) < 1e-7


def test_schulz_with_tolerance_converges():
    """SchulzInvert with truncation at 1e-10 reaches the fixed-rank run's
    residual with no larger ranks."""
    fx = load("c1")
    plain = build(D, fx, ctx_for(fx, 0.0))
    its_p, tr_p = plain.SchulzInvert(-1, 1.5, 6.0, 1e-5)
    c = ctx_for(fx, 1e-10)
    X = build(D, fx, c)
    its_t, tr_t = X.SchulzInvert(-1, 1.5, 6.0, 1e-5)
    assert tr_t[-1] < 1e-5 and abs(its_t - its_p) <= 1
    assert X.BlockCensus()["rank_sum"] <= plain.BlockCensus()["rank_sum"]
    A = build(D, fx, c)
    P = np.random.default_rng(3).standard_normal((A.Width(), 4))
    res = relerr(X.Multiply(1.0, A.Multiply(1.0, P)), P)
    assert res < 1e-4


def test_dist_hmat_single_rank():
    """Single-rank DistHMat2d: products and SchulzInvert under the global
    CompressionTolerance (DistHMat semantics) equal the HMat2d ones run with
    the same tolerance on a context; HMat2d itself stays at fixed rank."""
    fx = load("c1")
    sizes = [int(s) for s in fx["sizes"]]
    L, r = int(fx["levels"]), int(fx["rank"])
    S = D.operators.stencil(sizes, fx["coef"], L)
    P = fx["probes"]
    old = D.CompressionTolerance()
    try:
        D.SetCompressionTolerance(1e-10)
        c1 = D.Context(0)
        c1.set_oversample(int(fx["oversample"]))
        A = D.DistHMat2d(S, L, r, True, *sizes, D.Teams(), ctx=c1)
        assert A.LocalHeight() == A.Height() and A.FirstLocalRow() == 0
        C = A.Multiply(1.0, A, multType=2)
        assert c1.compression_tolerance() == 0.0          # restored after the product
        assert relerr(C.Multiply(1.0, P), fx["hh_AA"]) < 1e-11
        A.SchulzInvert(6, 2, 1.5, 6.0, 1e-4)
        c2 = D.Context(0)
        c2.set_oversample(int(fx["oversample"]))
        c2.set_compression_tolerance(1e-10)
        B = D.HMat2d(S, L, r, True, *sizes, ctx=c2)
        B.Multiply(1.0, B)                                # same generator use as above
        B.SchulzInvert(6)
        assert relerr(A.Multiply(1.0, P), B.Multiply(1.0, P)) < 1e-12
    finally:
        D.SetCompressionTolerance(old)
