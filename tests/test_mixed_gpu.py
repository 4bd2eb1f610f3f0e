"""Mixed precision: H*H products in the low-precision phase (range samples on
the TF32 tensor cores, block roundings in FP32) and mixed-precision Schulz.

Tolerances.  A low-precision product of random factors is compared with the
FP64 product of the same inputs and generator stream: relative 1e-2 on probe
vectors.  TF32 samples keep an 11-bit significand (5e-4), and random factors
give every compressed block a slowly decaying spectrum, so the fixed-rank
truncation amplifies the sample perturbation by 1 / (relative gap at the
truncation rank); the FP32 roundings add about 1e-6.  Products whose blocks
have exact rank within the samples (sparse-built factors) agree to 1e-5.  Mixed Schulz must reach the same stop test as the FP64 run
(||I - X A|| estimate below stopTol, checked in FP64), in at most one extra
iteration, and its inverse applied to probe vectors must agree with the
FP64 method's to the attained residual's order (10 x stopTol)."""
import numpy as np
import pytest

import dmhm_b200 as D
from helpers import build, load, relerr

pytestmark = pytest.mark.gpu


def fresh_ctx(fx):
    c = D.Context(0)
    c.set_oversample(int(fx["oversample"]))
    return c


@pytest.mark.parametrize("case", ["c1", "ragged", "c3d"])
def test_low_precision_product(case):
    fx = load(case)
    P = fx["probes"]
    out = []
    for low in (False, True):
        c = fresh_ctx(fx)
        c.set_low_precision(low)
        A = build(D, fx, c)
        A.SetToRandom()
        B = build(D, fx, c, "coefB" if "coefB" in fx else "coef")
        B.SetToRandom()
        out.append(A.Multiply(0.25, B).Multiply(1.0, P))
    err = relerr(out[1], out[0])
    assert 0.0 < err < 1e-2   # really computed in low precision, and close


def test_low_precision_exact_blocks():
    """Sparse-built factors: every compressed block has exact rank <= the
    samples, so only the FP32 roundings' error remains."""
    fx = load("c1")
    P = fx["probes"]
    c = fresh_ctx(fx)
    c.set_low_precision(True)
    A = build(D, fx, c)
    assert relerr(A.Multiply(1.0, A).Multiply(1.0, P), fx["hh_AA"]) < 1e-5


def check_mixed(make, P, stop):
    c, X = make()
    n64, tr64 = X.SchulzInvert(-1, 1.5, 6.0, stop)
    assert tr64[-1] < stop
    c2, Xm = make()
    nm, low, trm = Xm.SchulzInvertMixed(-1, 1.5, 6.0, stop, 1e-2)
    assert low >= 1                  # early iterations ran in low precision
    assert nm <= n64 + 1
    assert trm[-1] < stop            # the FP64 stop test passed
    _, A = make()
    res = relerr(Xm.Multiply(1.0, A.Multiply(1.0, P)), P)
    res64 = relerr(X.Multiply(1.0, A.Multiply(1.0, P)), P)
    assert res < max(10 * res64, 10 * stop)
    assert relerr(Xm.Multiply(1.0, P), X.Multiply(1.0, P)) < 10 * stop


@pytest.mark.parametrize("case", ["c1", "ragged", "c3d"])
def test_mixed_schulz_reaches_fp64_accuracy(case):
    fx = load(case)

    def make():
        c = fresh_ctx(fx)
        return c, build(D, fx, c)

    check_mixed(make, fx["probes"], 1e-4)


def test_mixed_schulz_to_1e8():
    """64 x 64 five-point operator, maxRank 16: the stop test at 1e-8."""
    sizes = (64, 64)
    coef = D.operators.uniform_coefficients(sizes, 3)
    S = D.operators.stencil(sizes, coef, 4)

    def make():
        c = D.Context(0)
        c.set_oversample(4)
        return c, D.HMat2d(S, 4, 16, True, *sizes, ctx=c)

    P = np.random.default_rng(1).standard_normal((64 * 64, 3))
    check_mixed(make, P, 1e-8)


def test_mixed_schulz_fixed_iterations():
    """Without the stop test all but the last three iterations are low."""
    fx = load("c1")
    c = fresh_ctx(fx)
    X = build(D, fx, c)
    n, low, _ = X.SchulzInvertMixed(6, 1.5, 6.0, 1e-4, 1e-2)
    assert (n, low) == (6, 3)
    c.set_low_precision(False)


def test_switch_zero_is_fp64():
    fx = load("c1")
    P = fx["probes"]
    c = fresh_ctx(fx)
    X = build(D, fx, c)
    n, low, tr = X.SchulzInvertMixed(3, 1.5, 6.0, 1e-4, 0.0)
    assert (n, low) == (3, 0)
    assert relerr(X.Multiply(1.0, P), fx["schulz3"]) < 1e-8
