"""Tensor-core TF32 H-matrix x dense (FP32 accumulation) against the FP64
product, for both kernel forms (1 = tcgen05 kind::tf32, 2 = mma.sync m16n8k8
persistent tiles) and the autotuned choice.  Tolerance: relative 5e-3 in the
Frobenius norm (TF32 keeps an 11-bit significand; block sums accumulate in
FP32)."""
import ctypes as C

import numpy as np
import pytest

import dmhm_b200 as D
from dmhm_b200 import _lib
from helpers import build, load, relerr

pytestmark = pytest.mark.gpu
TOL = 5e-3


def tf32(H, alpha, X, beta, Y):
    import torch
    n, k = X.shape
    Xt = X.t().contiguous()
    Yt = Y.t().contiguous()
    torch.cuda.synchronize()
    _lib.check(_lib.lib().hm_multiply_dense_tf32(H.handle, alpha, C.c_void_p(Xt.data_ptr()), n,
                                                 beta, C.c_void_p(Yt.data_ptr()), n, k))
    return Yt.t()


def set_kernel(ctx, which):
    _lib.check(_lib.lib().hm_set_tf32_kernel(ctx.handle, which))


@pytest.mark.parametrize("which", [1, 2])
@pytest.mark.parametrize("case,k", [("c1", 1), ("c1", 4), ("c1", 64), ("ragged", 7), ("weak", 33),
                                    ("c3d", 16)])
def test_tf32_against_fp64(case, k, which):
    import torch
    fx = load(case)
    ctx = D.Context(0)
    set_kernel(ctx, which)
    H = build(D, fx, ctx)
    H.SetToRandom()
    N = H.Height()
    g = torch.Generator().manual_seed(k)
    X = torch.randn(N, k, generator=g, dtype=torch.float64).cuda()
    Y0 = torch.randn(N, k, generator=g, dtype=torch.float64).cuda()
    ref = H.Multiply(0.5, X.cpu().numpy(), -1.0, Y0.cpu().numpy())
    got = tf32(H, 0.5, X, -1.0, Y0.clone()).cpu().numpy()
    assert relerr(got, ref) < TOL


def test_tf32_bench_shape():
    import torch
    sizes = (128, 128)
    ctx = D.Context(0)
    S = D.operators.stencil(sizes, D.operators.uniform_coefficients(sizes, 2), 5)
    H = D.HMat2d(S, 5, 16, True, *sizes, ctx=ctx)
    H.SetToRandom()
    X = torch.randn(16384, 64, dtype=torch.float64, device="cuda")
    Y = torch.zeros(16384, 64, dtype=torch.float64, device="cuda")
    got = tf32(H, 1.0, X, 0.0, Y).cpu().numpy()
    ref = H.Multiply(1.0, X.cpu().numpy())
    assert relerr(got, ref) < TOL
    # stale copy check: the FP32 copy follows changes of the matrix
    H.Scale(2.0)
    got2 = tf32(H, 1.0, X, 0.0, Y).cpu().numpy()
    assert relerr(got2, 2.0 * ref) < TOL


@pytest.mark.parametrize("case,k", [("c1", 100), ("weak", 130), ("c3d", 65)])
def test_tf32_many_columns(case, k):
    """More than 64 columns: the persistent mma.sync form, whatever is asked."""
    import torch
    fx = load(case)
    ctx = D.Context(0)
    H = build(D, fx, ctx)
    H.SetToRandom()
    N = H.Height()
    g = torch.Generator().manual_seed(k)
    X = torch.randn(N, k, generator=g, dtype=torch.float64).cuda()
    Y0 = torch.randn(N, k, generator=g, dtype=torch.float64).cuda()
    ref = H.Multiply(2.0, X.cpu().numpy(), 0.5, Y0.cpu().numpy())
    for which in (0, 1, 2):
        set_kernel(ctx, which)
        got = tf32(H, 2.0, X, 0.5, Y0.clone()).cpu().numpy()
        assert relerr(got, ref) < TOL


def test_tf32_autotune():
    """The tuned choice is one of the two forms, kept per layout and column
    bucket, and the product it runs is right."""
    import torch
    sizes = (64, 64)
    ctx = D.Context(0)
    S = D.operators.stencil(sizes, D.operators.uniform_coefficients(sizes, 2), 5)
    H = D.HMat2d(S, 4, 16, True, *sizes, ctx=ctx)
    H.SetToRandom()
    N = H.Height()
    X = torch.randn(N, 48, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    w = C.c_int(-1)
    _lib.check(_lib.lib().hm_tf32_kernel_choice(H.handle, C.c_void_p(X.data_ptr()), N, 48,
                                                C.byref(w)))
    assert w.value in (1, 2)
    w2 = C.c_int(-1)
    _lib.check(_lib.lib().hm_tf32_kernel_choice(H.handle, C.c_void_p(X.data_ptr()), N, 40,
                                                C.byref(w2)))
    assert w2.value == w.value   # same bucket (33..64), no second tuning
    Y = torch.zeros(N, 48, dtype=torch.float64, device="cuda")
    got = tf32(H, 1.0, X, 0.0, Y).cpu().numpy()
    assert relerr(got, H.Multiply(1.0, X.cpu().numpy())) < TOL
