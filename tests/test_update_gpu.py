"""UpdateWith (A := alpha B + A by RoundedUpdate per low-rank block and
Update per dense block), SetToIdentity and Conjugate, against the oracle's
restatement of the same block operations and against exact identities.

Tolerances: exact cases (ranks fit, or the sum has exact low rank) 1e-12;
random factors whose sum is truncated to maxRank 1e-9 against the oracle,
as for the H*H products of random factors."""
import numpy as np
import pytest

import dmhm_b200 as D
from helpers import build, load, relerr

pytestmark = pytest.mark.gpu


def fresh_ctx(fx):
    c = D.Context(0)
    c.set_oversample(int(fx["oversample"]))
    return c


def test_update_with_exact():
    fx = load("c1")
    c = fresh_ctx(fx)
    P = fx["probes"]
    A = build(D, fx, c)
    A.SetToRandom()
    B = build(D, fx, c, "coefB")                   # sparse-built: rank-0 admissible blocks
    ref = A.Multiply(1.0, P) + 0.5 * B.Multiply(1.0, P)
    A.UpdateWith(0.5, B)
    assert relerr(A.Multiply(1.0, P), ref) < 1e-13
    # a sum of exact rank maxRank through the rounding path: A + (-0.25) A
    B2 = D.HMat2d(ctx=c).CopyFrom(A)
    ref2 = 0.75 * A.Multiply(1.0, P)
    A.UpdateWith(-0.25, B2)
    assert relerr(A.Multiply(1.0, P), ref2) < 1e-12


@pytest.mark.parametrize("case", ["c1", "ragged"])
def test_update_with_random_against_oracle(case):
    from oracle import dmhm_oracle as O
    fx = load(case)
    sizes = tuple(int(s) for s in fx["sizes"])
    L, r = int(fx["levels"]), int(fx["rank"])
    c = fresh_ctx(fx)
    A = build(D, fx, c)
    A.SetToRandom()
    B = build(D, fx, c, "coefB")
    B.SetToRandom()
    A.UpdateWith(0.3, B)
    rng = O.Rng(int(fx["oversample"]))
    Ao = O.build_stencil_hmat(2, sizes, L, r, fx["coef"], strong=bool(fx["strong"]))
    O.set_to_random(Ao, rng)
    Bo = O.build_stencil_hmat(2, sizes, L, r, fx["coefB"], strong=bool(fx["strong"]))
    O.set_to_random(Bo, rng)
    for a, b in zip(Ao.leaves(), Bo.leaves()):
        if a.kind == O.DENSE:
            a.D = a.D + 0.3 * b.D
        else:
            F = O.rounded_update(r, 0.3, O.LR(b.U, b.V), 1.0, O.LR(a.U, a.V))
            a.U, a.V = F.U, F.V
    P = fx["probes"]
    assert relerr(A.Multiply(1.0, P), O.multiply_dense(Ao, 1.0, P)) < 1e-9


def test_set_to_identity_and_conjugate():
    fx = load("ragged")
    c = fresh_ctx(fx)
    P = fx["probes"]
    A = build(D, fx, c)
    A.SetToRandom()
    A.SetToIdentity()
    assert A.BlockCensus()["rank_sum"] == 0
    assert relerr(A.Multiply(1.0, P), P) < 1e-15
    B = build(D, fx, c)
    ref = B.Multiply(1.0, P)
    B.Conjugate()                                  # real: nothing changes
    assert np.array_equal(B.Multiply(1.0, P), ref)
