"""One low-rank approximation of a whole product (hmat_tools::Multiply,
TransposeMultiply, AdjointMultiply: F := alpha op(A) B by the randomized range
finder) against the reference's own F (tests/golden fixtures made by the
compiled reference) on probe vectors.

The test matrices are the reference's draws (same serial generator position
on a fresh context), so F agrees to rounding where the rank-r truncation is
well separated; tolerance 1e-9 relative, as for the H*H products of random
factors."""
import numpy as np
import pytest

import dmhm_b200 as D
from dmhm_b200 import _lib
from helpers import build, load, relerr

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["c1", "ragged"])
@pytest.mark.parametrize("op,tag", [(0, "lr_AB"), (1, "lr_AtB"), (2, "lr_AtB")])
def test_low_rank_product_matches_reference(case, op, tag):
    fx = load(case)
    c = D.Context(0)
    c.set_oversample(int(fx["oversample"]))
    A = build(D, fx, c)
    A.SetToRandom()
    B = build(D, fx, c, "coefB")
    U, V = A.LowRankProduct(0.75, B, int(fx["rank"]) + int(fx["oversample"]), op)
    assert U.shape[1] == int(fx[tag + "_rank"])
    P = fx["probes"]
    assert relerr(U @ (V.T @ P), fx[tag]) < 1e-9
    # the generator advanced by one n x sampleRank fill
    n = A.Height()
    s = int(fx["rank"]) + int(fx["oversample"])
    from oracle import dmhm_oracle as O
    am, cm = O.lcg_jump(s * 2 * ((n + 1) // 2))
    assert c.lcg_states()[0] == (am * O.LCG_SEED + cm) % (1 << 64)


def test_low_rank_product_errors():
    fx = load("c1")
    c = D.Context(0)
    A = build(D, fx, c)
    with pytest.raises(_lib.HMError):
        A.LowRankProduct(1.0, A, A.Height() + 1)       # more samples than rows
    with pytest.raises(_lib.HMError):
        A.LowRankProduct(1.0, A, 8, op=3)
