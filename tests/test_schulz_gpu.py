"""Schulz inversion and two-norm estimation on the GPU against the reference.

Tolerances: the norm estimate to 1e-12 (a power method with the same start
vector); the inverse applied to probe vectors to 1e-8 after 2-3 iterations
and to 1e-6 after the full 13-iteration stop-tested run, because each
iteration's fixed-rank truncations amplify rounding differences."""
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
def test_two_norm_estimate(case):
    fx = load(case)
    c = fresh_ctx(fx)
    A = build(D, fx, c)
    key = "schulz2_trace" if case == "c3d" else "schulz3_trace"
    est = D.EstimateTwoNorm(A, 1.5, 6.0)
    assert abs(est - fx[key][0]) < 1e-12 * est


@pytest.mark.parametrize("case,its", [("c1", 3), ("ragged", 3), ("weak", 3), ("c3d", 2)])
def test_fixed_iterations(case, its):
    fx = load(case)
    c = fresh_ctx(fx)
    A = build(D, fx, c)
    n, trace = A.SchulzInvert(its)
    assert n == its
    key = f"schulz{its}"
    assert abs(trace[0] - fx[key + "_trace"][0]) < 1e-12 * trace[0]
    assert relerr(A.Multiply(1.0, fx["probes"]), fx[key]) < 1e-8


def test_stop_tested_run_matches_reference():
    fx = load("c1")
    c = fresh_ctx(fx)
    A = build(D, fx, c)
    n, trace = A.SchulzInvert(-1, 1.5, 6.0, 1e-4)
    ref_trace = fx["schulz_stop_trace"]
    assert n == int(fx["schulz_stop_iterations"])
    assert len(trace) == len(ref_trace)
    # estimates of ||I - X_k A|| are compared absolutely (they measure a
    # deviation from the identity, whose norm is 1)
    np.testing.assert_allclose(trace, ref_trace, rtol=1e-5, atol=1e-7)
    assert relerr(A.Multiply(1.0, fx["probes"]), fx["schulz_stop"]) < 1e-6
