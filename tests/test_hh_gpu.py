"""H*H product with randomized compression on the GPU against the reference
fixtures and the numpy oracle.

The test matrices of the sampled products come from the same generator
stream as the reference's, so the compressed blocks agree to rounding where
the truncation is well conditioned.  Tolerances (relative, Frobenius norm of
C applied to probe vectors): 1e-12 for products whose compressed blocks are
exact (sparse-built factors), 1e-9 where fixed-rank truncation discards
content (random factors)."""
import numpy as np
import pytest

import dmhm_b200 as D
from helpers import build, load, relerr

pytestmark = pytest.mark.gpu


def fresh_ctx(fx):
    c = D.Context(0)
    c.set_oversample(int(fx["oversample"]))
    return c


@pytest.mark.parametrize("case", ["c1", "ragged", "weak", "c3d"])
def test_square_matches_reference(case):
    fx = load(case)
    c = fresh_ctx(fx)
    A = build(D, fx, c)
    Cm = A.Multiply(1.0, A)
    assert relerr(Cm.Multiply(1.0, fx["probes"]), fx["hh_AA"]) < 1e-12


@pytest.mark.parametrize("case", ["c1", "ragged"])
def test_general_matches_reference(case):
    fx = load(case)
    c = fresh_ctx(fx)
    A = build(D, fx, c)
    B = build(D, fx, c, "coefB")
    Cm = A.Multiply(-0.5, B)
    assert relerr(Cm.Multiply(1.0, fx["probes"]), fx["hh_AB"]) < 1e-12


def test_generator_advances_like_reference():
    """Same number of serial draws as the oracle's recursion."""
    from oracle import dmhm_oracle as O
    fx = load("ragged")
    c = fresh_ctx(fx)
    A = build(D, fx, c)
    A.Multiply(1.0, A)
    rng = O.Rng(int(fx["oversample"]))
    Ao = O.build_stencil_hmat(2, (24, 20), 3, 6, fx["coef"])
    O.hh_multiply(Ao, 1.0, Ao, rng)
    assert c.lcg_states()[0] == rng.serial.state


@pytest.mark.parametrize("case", ["c1", "ragged", "weak"])
def test_random_factors_against_oracle(case):
    from oracle import dmhm_oracle as O
    fx = load(case)
    sizes = tuple(int(s) for s in fx["sizes"])
    L, r = int(fx["levels"]), int(fx["rank"])
    c = fresh_ctx(fx)
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
    Co = O.hh_multiply(Ao, 0.25, Bo, rng)
    P = fx["probes"]
    assert relerr(Cm.Multiply(1.0, P), O.multiply_dense(Co, 1.0, P)) < 1e-9
    # and the update form C :~= alpha A B + beta C
    Cm2 = A.Multiply(1.0, B, 0.5, Cm)
    O.hh_multiply_update(Ao, 1.0, Bo, 0.5, Co, rng)
    assert relerr(Cm2.Multiply(1.0, P), O.multiply_dense(Co, 1.0, P)) < 1e-9


def test_copy_transpose_scale_diagonal(ctx):
    from oracle import dmhm_oracle as O
    fx = load("ragged")
    c = fresh_ctx(fx)
    A = build(D, fx, c)
    A.SetToRandom()
    Ao = O.build_stencil_hmat(2, (24, 20), 3, 6, fx["coef"])
    O.set_to_random(Ao, O.Rng())
    P = fx["probes"]
    X = D.HMat2d(ctx=c).AdjointFrom(A)
    assert relerr(X.Multiply(1.0, P), O.transpose_multiply_dense(Ao, 1.0, P)) < 1e-14
    X.Scale(-2.0)
    X.AddConstantToDiagonal(3.0)
    ref = -2.0 * O.transpose_multiply_dense(Ao, 1.0, P) + 3.0 * P
    assert relerr(X.Multiply(1.0, P), ref) < 1e-14
    Y = D.HMat2d(ctx=c).CopyFrom(X)
    assert relerr(Y.Multiply(1.0, P), ref) < 1e-15


def test_errors():
    fx = load("weak")
    c = fresh_ctx(fx)
    A = build(D, fx, c)
    with pytest.raises(D.HMError):
        A.Multiply(1.0, A, 1.0, A)          # C aliases a factor
    other = load("ragged")
    B = build(D, other, c)
    with pytest.raises(D.HMError):
        A.Multiply(1.0, B)                  # different structures


@pytest.mark.parametrize("case", ["c1", "c3d"])
def test_cached_lists_replay(case):
    """The second product with the same plan replays the cached
    position-independent block lists against new buffers: same generator
    state, same result, also when the factors change from A * A to A * B
    with the same ranks."""
    fx = load(case)
    P = fx["probes"]
    c = fresh_ctx(fx)
    A = build(D, fx, c)
    A.SetToRandom()
    B = build(D, fx, c, "coefB" if "coefB" in fx else "coef")
    B.SetToRandom()
    st = c.lcg_states()
    C1 = A.Multiply(0.5, B).Multiply(1.0, P)
    c.set_lcg_states(*st)
    C2 = A.Multiply(0.5, B).Multiply(1.0, P)
    assert np.array_equal(C1, C2)
    c.set_lcg_states(*st)
    AA1 = A.Multiply(0.5, A).Multiply(1.0, P)
    c.set_lcg_states(*st)
    AA2 = A.Multiply(0.5, A).Multiply(1.0, P)
    assert np.array_equal(AA1, AA2)
    # a fresh context (no cached lists) agrees with the replays
    c2 = fresh_ctx(fx)
    A2 = build(D, fx, c2)
    A2.SetToRandom()
    B2 = build(D, fx, c2, "coefB" if "coefB" in fx else "coef")
    B2.SetToRandom()
    c2.set_lcg_states(*st)
    assert np.array_equal(A2.Multiply(0.5, B2).Multiply(1.0, P), C1)
