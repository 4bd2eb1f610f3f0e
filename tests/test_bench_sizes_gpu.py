"""Parity at the benchmark workloads' own sizes, against outputs of the
reference library (tests/golden/make_golden.py, cases cfg1s, cfg2, cfg3,
cfg4).  Inputs are regenerated from the fixtures' hash seeds; outputs are
compared on a few full columns and on a sketch G^T Y of every column.

Tolerances:
* H x 64 right-hand sides (FP64) and its transpose: 1e-13 relative, the
  matvec tolerance (only the summation order differs from the reference);
* the TF32 form of the same product: 1e-3 relative (TF32 keeps 10 mantissa
  bits of each input);
* A A of the 32^3 operator: 1e-12 (the product is exact, only rounding);
* SchulzInvert on the 32^2 operator to stopTol 1e-8 (30 iterations, the
  reference's cap, without reaching the tolerance): the iteration count
  exactly; the norm estimates to rtol 1e-4 / atol 1e-6, and below 1e-6
  (both runs) at the floor the fixed rank 8 leaves (||I - X A|| about 3e-7
  from iteration 14 on, where the estimates are rounding noise of that
  size); X P to 1e-5, an order above that floor (fixed-rank truncations
  amplify rounding differences from one iteration to the next);
* two SchulzInvert iterations on the 256^2 log-uniform operator: the
  initial norm estimate to 1e-12 and X P to 1e-8, the fixed-iteration
  tolerances of the small cases.
"""
import numpy as np
import pytest

import dmhm_b200 as D
from helpers import big_case_inputs, load, relerr

pytestmark = pytest.mark.gpu


def _operator(fx, ctx):
    sizes = [int(s) for s in fx["sizes"]]
    L = int(fx["levels"])
    coef, X, G = big_case_inputs(fx)
    S = D.operators.stencil(sizes, coef, L)
    cls = D.HMat2d if len(sizes) == 2 else D.HMat3d
    return cls(S, L, int(fx["rank"]), True, *sizes, ctx=ctx), X, G


def _tf32(H, X):
    import ctypes as C

    import torch
    from dmhm_b200 import _lib
    n, k = X.shape
    Xt = torch.tensor(X.T.copy(), device="cuda")          # column-major n x k
    Yt = torch.zeros((k, n), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    _lib.check(_lib.lib().hm_multiply_dense_tf32(H.handle, 1.0, C.c_void_p(Xt.data_ptr()), n,
                                                 0.0, C.c_void_p(Yt.data_ptr()), n, k))
    torch.cuda.synchronize()
    return Yt.cpu().numpy().T


def _check(fx, tag, Y, G, tol):
    keep = fx[tag].shape[1]
    assert relerr(Y[:, :keep], fx[tag]) < tol
    assert relerr(G.T @ Y, fx[tag + "_sketch"]) < tol


def test_cfg2_matmat_64_rhs():
    fx = load("cfg2")
    ctx = D.Context(0)                  # fresh generators, as after Initialize
    ctx.set_oversample(int(fx["oversample"]))
    H, X, G = _operator(fx, ctx)
    H.SetToRandom()
    assert X.shape == (16384, 64)
    _check(fx, "Y", H.Multiply(1.0, X), G, 1e-13)
    _check(fx, "YT", H.TransposeMultiply(1.0, X), G, 1e-13)
    # one vector through the HBM-bound kernels
    y1 = H.Multiply(1.0, X[:, 0])
    assert relerr(y1, fx["Y"][:, 0]) < 1e-13
    # the TF32 tensor-core form of the same product (autotuned kernel form)
    Y32 = _tf32(H, X)
    assert relerr(Y32[:, :fx["Y"].shape[1]], fx["Y"]) < 1e-3
    assert relerr(G.T @ Y32, fx["Y_sketch"]) < 1e-3


def test_cfg3_hh_32cubed():
    fx = load("cfg3")
    ctx = D.Context(0)
    ctx.set_oversample(int(fx["oversample"]))
    A, X, G = _operator(fx, ctx)
    C = A.Multiply(1.0, A)
    _check(fx, "CP", C.Multiply(1.0, X), G, 1e-12)


def test_cfg1_schulz_to_1e8():
    fx = load("cfg1s")
    ctx = D.Context(0)
    ctx.set_oversample(int(fx["oversample"]))
    A, X, G = _operator(fx, ctx)
    n, trace = A.SchulzInvert(int(fx["iters"]), 1.5, 6.0, float(fx["stopTol"]))
    assert n == int(fx["iterations"])
    ref = np.asarray(fx["trace"])
    trace = np.asarray(trace)
    assert trace.shape == ref.shape
    # while converging, every estimate agrees to rtol 1e-4; at the method's
    # floor (fixed rank 8: ||I - X A|| stalls near 3e-7 from iteration 14
    # on) the estimates are rounding noise of that size, compared absolutely
    np.testing.assert_allclose(trace, ref, rtol=1e-4, atol=1e-6)
    floor = ref < 1e-5
    assert np.all(trace[floor] < 1e-6) and np.all(ref[floor] < 1e-6)
    xp = A.Multiply(1.0, X)
    err = relerr(xp[:, :fx["XP"].shape[1]], fx["XP"])
    print(f"cfg1s: X P relerr {err:.2e}, final estimates {trace[-1]:.2e} / {ref[-1]:.2e}")
    _check(fx, "XP", xp, G, 1e-5)


def test_cfg4_schulz_two_iterations_256():
    fx = load("cfg4")
    ctx = D.Context(0)
    ctx.set_oversample(int(fx["oversample"]))
    A, X, G = _operator(fx, ctx)
    n, trace = A.SchulzInvert(int(fx["iters"]))
    assert n == int(fx["iters"])
    assert abs(trace[0] - fx["trace"][0]) < 1e-12 * trace[0]
    _check(fx, "XP", A.Multiply(1.0, X), G, 1e-8)
