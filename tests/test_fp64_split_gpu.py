"""FP64 products of 9 to 16 columns: one pass of the tensor-core tiles or
8-column passes of the streaming kernels, chosen by timing (hm_set_fp64_split
0) or forced (1, 2).  Every choice must give the oracle's product (the
reference's MultiplyDense, src/HMat2d/MultiplyDense-incl.hpp:12-68) to the
H x dense tolerance, with beta applied once per column."""
import ctypes as C

import numpy as np
import pytest

import dmhm_b200 as D
from dmhm_b200 import _lib
from helpers import build, load, relerr

pytestmark = pytest.mark.gpu
TOL = 1e-13


@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("k", [9, 12, 16])
def test_split_modes_against_oracle(mode, k):
    import torch
    from oracle import dmhm_oracle as O
    fx = load("c1")
    c = D.Context(0)
    _lib.check(_lib.lib().hm_set_fp64_split(c.handle, mode))
    H = build(D, fx, c)
    H.SetToRandom()
    Ho = O.build_stencil_hmat(2, (32, 32), 4, 8, fx["coef"])
    O.set_to_random(Ho, O.Rng())
    rng = np.random.default_rng(100 + k)
    X = rng.standard_normal((1024, k))
    Y0 = rng.standard_normal((1024, k))
    assert relerr(H.Multiply(1.0, X), O.multiply_dense(Ho, 1.0, X)) < TOL
    assert relerr(H.TransposeMultiply(2.0, X), O.transpose_multiply_dense(Ho, 2.0, X)) < TOL
    # C := alpha H X + beta C through the C ABI (device buffers)
    Xd = torch.tensor(X.T.copy(), device="cuda")
    Yd = torch.tensor(Y0.T.copy(), device="cuda")
    _lib.check(_lib.lib().hm_multiply_dense(H.handle, 0, 0.5, C.c_void_p(Xd.data_ptr()), 1024,
                                            -1.5, C.c_void_p(Yd.data_ptr()), 1024, k))
    c.synchronize()
    ref = 0.5 * O.multiply_dense(Ho, 1.0, X) - 1.5 * Y0
    assert relerr(Yd.cpu().numpy().T, ref) < TOL
    which = C.c_int()
    _lib.check(_lib.lib().hm_fp64_split_choice(H.handle, C.c_void_p(Xd.data_ptr()), 1024, k,
                                               C.byref(which)))
    assert which.value in (1, 2)
    if mode:
        assert which.value == mode
