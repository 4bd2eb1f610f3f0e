"""The allocation-free H-matrix x vector entry point, hm_multiply_vector_noalloc.

Callers whose memory manager already owns the GPU's memory, or whose
time-critical loops must not call the allocator, use this variant: it keeps
its intermediates in a static device array instead of allocating.  Checked
through the C ABI against hm_multiply_dense (same tolerance as the other
H-matvec tests) on two calls in a row, since the static array keeps the
previous call's contents.  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

import dmhm_b200 as D
from dmhm_b200 import _lib
from helpers import build, load, relerr

pytestmark = pytest.mark.gpu
TOL = 1e-13


def _noalloc(H, trans, alpha, x, beta, y):
    _lib.check(_lib.lib().hm_multiply_vector_noalloc(
        H.handle, trans, alpha, C.c_void_p(x.data_ptr()), beta, C.c_void_p(y.data_ptr())))


def _existing(H, trans, alpha, x, beta, y):
    n = x.shape[0]
    m = y.shape[0]
    _lib.check(_lib.lib().hm_multiply_dense(
        H.handle, trans, alpha, C.c_void_p(x.data_ptr()), n, beta, C.c_void_p(y.data_ptr()),
        m, 1))


@pytest.mark.parametrize("case", ["c1", "ragged", "weak", "c3d"])
def test_noalloc_matches_existing_twice(case):
    import torch
    fx = load(case)
    ctx = D.Context(0)
    H = build(D, fx, ctx)
    H.SetToRandom()
    N = H.Height()
    g = torch.Generator(device="cpu").manual_seed(7)
    for trans in (0, 1):
        for call in range(2):          # two calls in a row share the static scratch
            x = torch.randn(N, generator=g, dtype=torch.float64).cuda()
            y0 = torch.randn(N, generator=g, dtype=torch.float64).cuda()
            alpha, beta = 1.5 - call, 0.25 * call
            y_new, y_ref = y0.clone(), y0.clone()
            _noalloc(H, trans, alpha, x, beta, y_new)
            _existing(H, trans, alpha, x, beta, y_ref)
            ctx.synchronize()
            assert relerr(y_new.cpu().numpy(), y_ref.cpu().numpy()) < TOL, (case, trans, call)


def test_noalloc_rejects_oversized_matrix():
    import torch
    ctx = D.Context(0)
    sizes = (256, 256)
    S = D.operators.stencil(sizes, D.operators.uniform_coefficients(sizes, 3), 6)
    H = D.HMat2d(S, 6, 16, True, *sizes, ctx=ctx)
    H.SetToRandom()                    # ~31920 blocks at rank 16: > 4 MiB of scratch
    x = torch.zeros(H.Width(), dtype=torch.float64, device="cuda")
    y = torch.zeros(H.Height(), dtype=torch.float64, device="cuda")
    with pytest.raises(D.HMError) as e:
        _noalloc(H, 0, 1.0, x, 0.0, y)
    assert e.value.status == 4 and "static scratch" in str(e.value)
