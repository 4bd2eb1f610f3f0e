"""DirectInvert (recursive Schur complements, src/HMat2d/Invert-incl.hpp:
17-125 and src/HMat3d/Invert-incl.hpp:14-122) on the GPU against the
reference's own DirectInvert applied to the fixture probes.

Tolerance: 1e-8 relative on the probes.  The reference's block products
truncate to the fixed rank maxRank after randomized compressions; the
engine draws the same samples in the same order, so the results differ only
by the rounding of the two SVD implementations, amplified through the
recursion's products."""
import time

import numpy as np
import pytest

import dmhm_b200 as D
from helpers import build, load, relerr

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["c1", "ragged", "weak", "c3d"])
def test_direct_invert_matches_reference(case):
    fx = load(case)
    ctx = D.Context(0)                    # generators as after Initialize
    ctx.set_oversample(int(fx["oversample"]))
    A = build(D, fx, ctx)
    t0 = time.perf_counter()
    A.DirectInvert()
    ctx.synchronize()
    secs = time.perf_counter() - t0
    got = A.Multiply(1.0, fx["probes"])
    err = relerr(got, fx["direct"])
    print(f"{case}: DirectInvert {secs:.3f} s (reference {float(fx['direct_seconds']):.3f} s), "
          f"relerr {err:.2e}")
    assert err < 1e-8


def test_direct_invert_is_an_inverse_and_keeps_the_context_usable():
    fx = load("c1")
    ctx = D.Context(0)
    ctx.set_oversample(int(fx["oversample"]))
    A = build(D, fx, ctx)
    X = build(D, fx, ctx)
    X.DirectInvert()
    P = fx["probes"]
    # X A p ~= p to the accuracy of the fixed-rank products (maxRank 8)
    res = np.linalg.norm(X.Multiply(1.0, A.Multiply(1.0, P)) - P) / np.linalg.norm(P)
    assert res < 1e-4
    # a compression tolerance on the context does not change the fixed-rank
    # method (as the reference's HMat2d ignores CompressionTolerance) and is
    # restored afterwards
    c2 = D.Context(0)
    c2.set_oversample(int(fx["oversample"]))
    c2.set_compression_tolerance(1e-6)
    Y = build(D, fx, c2)
    Y.DirectInvert()
    assert c2.compression_tolerance() == 1e-6
    assert relerr(Y.Multiply(1.0, P), fx["direct"]) < 1e-8
