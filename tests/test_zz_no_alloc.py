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


def test_noalloc_variable_ranks_alternating_matrices():
    """Two matrices of different layouts in alternation: the sparse-built
    operator (every admissible block of rank 0) and a Schulz inverse truncated
    by a compression tolerance (ranks from 1 up to maxRank); the last call has beta = 0 with
    a NaN-filled y, which must be overwritten, not scaled."""
    import torch
    fx = load("c1")
    ctx = D.Context(0)
    A = build(D, fx, ctx)
    Cm = build(D, fx, ctx)
    ctx.set_compression_tolerance(1e-6)
    Cm.SchulzInvert(4)                 # an approximate inverse stored at the ranks kept
    ctx.set_compression_tolerance(0.0)
    ranks = Cm.BlockCensus()
    assert ranks["rank_sum"] < ranks["low_rank"] * int(fx["rank"])    # ranks vary
    N = A.Height()
    g = torch.Generator(device="cpu").manual_seed(11)
    for call, H in enumerate((A, Cm, A, Cm)):
        x = torch.randn(N, generator=g, dtype=torch.float64).cuda()
        y0 = torch.randn(N, generator=g, dtype=torch.float64).cuda()
        beta = 0.5 if call < 3 else 0.0
        if call == 3:
            y0.fill_(float("nan"))
        y_new, y_ref = y0.clone(), y0.clone()
        _noalloc(H, call % 2, 0.75, x, beta, y_new)
        _existing(H, call % 2, 0.75, x, beta, y_ref)
        ctx.synchronize()
        assert torch.isfinite(y_new).all()
        assert relerr(y_new.cpu().numpy(), y_ref.cpu().numpy()) < TOL, call


def test_noalloc_rejects_oversized_matrix():
    import torch
    ctx = D.Context(0)
    sizes = (256, 256)
    S = D.operators.stencil(sizes, D.operators.uniform_coefficients(sizes, 3), 6)
    H = D.HMat2d(S, 6, 32, True, *sizes, ctx=ctx)
    H.SetToRandom()                    # ~31920 blocks at rank 32: about twice the 4 MiB
    x = torch.zeros(H.Width(), dtype=torch.float64, device="cuda")
    y = torch.zeros(H.Height(), dtype=torch.float64, device="cuda")
    with pytest.raises(D.HMError) as e:
        _noalloc(H, 0, 1.0, x, 0.0, y)
    assert e.value.status == 4 and "static scratch" in str(e.value)
