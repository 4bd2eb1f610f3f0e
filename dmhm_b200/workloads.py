"""Standard single-GPU workloads of the library, for timing and profiling.

    python -m dmhm_b200.workloads matmul [k]   # 128 x 128 operator, k-column H x dense (k = 64)
    python -m dmhm_b200.workloads matvec       # the same operator, one vector, four products
    python -m dmhm_b200.workloads tf32 [k]     # TF32 H x dense, mma.sync form, three products
    python -m dmhm_b200.workloads schulz64 [n] # SchulzInvert(n = 3) on the 64 x 64 operator
    python -m dmhm_b200.workloads direct       # DirectInvert on the 32 x 32 operator
    python -m dmhm_b200.workloads hh3d [n]     # n (= 3) products A A of the 32^3 operator

The 128 x 128 operator is the five-point grid operator (c ~ U[1, 2), seed
2), numLevels 5 (64-point leaves), maxRank 16, strong admissibility, every
admissible block at full rank (SetToRandom): 275.6 MB of block data, more than
the 126 MB L2.  The 64 x 64 Schulz case has numLevels 4, maxRank 16 and
oversample 4.  Each workload builds its operator, runs its products and
prints "done"; run it under a profiler with a kernel filter and a launch
skip count to capture one steady-state launch.
"""
from __future__ import annotations

import ctypes as C
import sys

import numpy as np

from . import _lib
from . import operators
from .hmat import Context, HMat2d


def _operator_128(ctx):
    sizes = (128, 128)
    S = operators.stencil(sizes, operators.uniform_coefficients(sizes, 2), 5)
    H = HMat2d(S, 5, 16, True, *sizes, ctx=ctx)
    H.SetToRandom()
    return H


def _device_blocks(N, k):
    """Column-major N x k input (standard normal, seed 3) and output on the
    device (torch owns the memory; the library only reads the pointers)."""
    import torch
    x = np.random.default_rng(3).standard_normal((k, N))
    X = torch.tensor(x, dtype=torch.float64, device="cuda")
    Y = torch.zeros((k, N), dtype=torch.float64, device="cuda")
    return X, Y


def matmul(k: int = 64, products: int = 3):
    """Y = H X through hm_multiply_dense (FP64; k <= 8 takes the few-column
    streaming kernels, wider blocks the FP64 tensor-core kernels)."""
    ctx = Context(0)
    H = _operator_128(ctx)
    N = H.Height()
    X, Y = _device_blocks(N, k)
    lib = _lib.lib()
    for _ in range(products):
        _lib.check(lib.hm_multiply_dense(H.handle, 0, 1.0, C.c_void_p(X.data_ptr()), N, 0.0,
                                         C.c_void_p(Y.data_ptr()), N, k))
    ctx.synchronize()


def tf32(k: int = 64, products: int = 3):
    """Y = H X through hm_multiply_dense_tf32 with the mma.sync form forced."""
    ctx = Context(0)
    H = _operator_128(ctx)
    N = H.Height()
    X, Y = _device_blocks(N, k)
    lib = _lib.lib()
    _lib.check(lib.hm_set_tf32_kernel(ctx.handle, 2))
    for _ in range(products):
        _lib.check(lib.hm_multiply_dense_tf32(H.handle, 1.0, C.c_void_p(X.data_ptr()), N, 0.0,
                                              C.c_void_p(Y.data_ptr()), N, k))
    ctx.synchronize()


def schulz64(iterations: int = 3):
    """SchulzInvert(iterations) on the 64 x 64 operator (numLevels 4,
    maxRank 16, oversample 4)."""
    sizes = (64, 64)
    ctx = Context(0)
    ctx.set_oversample(4)
    S = operators.stencil(sizes, operators.uniform_coefficients(sizes, 2), 4)
    H = HMat2d(S, 4, 16, True, *sizes, ctx=ctx)
    H.SchulzInvert(iterations)
    ctx.synchronize()


def direct():
    """DirectInvert on the 32 x 32 operator (numLevels 4: 16-point leaves,
    maxRank 8, oversample 4)."""
    sizes = (32, 32)
    ctx = Context(0)
    ctx.set_oversample(4)
    S = operators.stencil(sizes, operators.uniform_coefficients(sizes, 2), 4)
    H = HMat2d(S, 4, 8, True, *sizes, ctx=ctx)
    H.DirectInvert()
    ctx.synchronize()


def hh3d(products: int = 3):
    """C = A A for the 32 x 32 x 32 seven-point operator (c ~ U[1, 2), seed
    3; numLevels 4: 64-point leaves, maxRank 24, oversample 8, compression
    tolerance 1e-10), `products` times."""
    from .hmat import HMat3d
    sizes = (32, 32, 32)
    ctx = Context(0)
    ctx.set_oversample(8)
    ctx.set_compression_tolerance(1e-10)
    S = operators.stencil(sizes, operators.uniform_coefficients(sizes, 3), 4)
    A = HMat3d(S, 4, 24, True, *sizes, ctx=ctx)
    for _ in range(products):
        C_ = A.Multiply(1.0, A)
        ctx.synchronize()
        del C_


def main(argv):
    case = argv[0] if argv else "matmul"
    arg = int(argv[1]) if len(argv) > 1 else None
    if case == "matmul":
        matmul(arg or 64)
    elif case == "matvec":
        matmul(1, products=4)
    elif case == "tf32":
        tf32(arg or 64)
    elif case == "schulz64":
        schulz64(arg or 3)
    elif case == "direct":
        direct()
    elif case == "hh3d":
        hh3d(arg or 3)
    else:
        raise SystemExit(f"unknown workload {case}")
    print("done")


if __name__ == "__main__":
    main(sys.argv[1:])
