"""H-matrix x vector / dense on the GPU against the reference fixtures and
the numpy oracle (tolerance: relative 1e-13 in the Frobenius norm; the
accumulation order differs from the reference's recursion)."""
import numpy as np
import pytest

import dmhm_b200 as D
from helpers import build, load, relerr

pytestmark = pytest.mark.gpu
CASES = ["c1", "ragged", "weak", "c3d"]
TOL = 1e-13


@pytest.mark.parametrize("case", CASES)
def test_matvec_matches_reference(ctx, case):
    fx = load(case)
    H = build(D, fx, ctx)
    P = fx["probes"]
    assert relerr(H.Multiply(1.0, P), fx["matvec"]) < TOL
    assert relerr(H.Multiply(1.0, P[:, 0]), fx["matvec1"]) < TOL
    assert relerr(H.TransposeMultiply(1.0, P), fx["matvec_T"]) < TOL


@pytest.mark.parametrize("case", CASES)
def test_random_matvec_matches_reference(ctx, case):
    fx = load(case)
    c = D.Context(0)            # fresh generators, as after Initialize
    H = build(D, fx, c)
    H.SetToRandom()
    P = fx["probes"]
    assert relerr(H.Multiply(1.0, P), fx["random"]) < TOL
    assert relerr(H.TransposeMultiply(1.0, P), fx["random_T"]) < TOL
    assert relerr(H.Multiply(1.0, P[:, 0]), fx["random"][:, 0]) < TOL


def test_alpha_beta_and_device_tensors(ctx):
    import torch
    fx = load("ragged")
    H = build(D, fx, ctx)
    H.SetToRandom()
    P = fx["probes"]
    Y0 = np.random.default_rng(3).standard_normal(P.shape)
    ref = -0.7 * H.Multiply(1.0, P) + 0.3 * Y0
    got = H.Multiply(-0.7, P, 0.3, Y0)
    assert relerr(got, ref) < TOL
    Pt = torch.tensor(P, device="cuda")
    Yt = H.Multiply(1.0, Pt)
    assert Yt.is_cuda
    assert relerr(Yt.cpu().numpy(), H.Multiply(1.0, P)) < TOL


@pytest.mark.parametrize("k", [1, 2, 5, 8, 9, 40, 64, 100])
def test_widths_against_oracle(ctx, k):
    from oracle import dmhm_oracle as O
    fx = load("c1")
    c = D.Context(0)
    H = build(D, fx, c)
    H.SetToRandom()
    Ho = O.build_stencil_hmat(2, (32, 32), 4, 8, fx["coef"])
    O.set_to_random(Ho, O.Rng())
    X = np.random.default_rng(k).standard_normal((1024, k))
    assert relerr(H.Multiply(1.0, X), O.multiply_dense(Ho, 1.0, X)) < TOL
    assert relerr(H.TransposeMultiply(2.0, X), O.transpose_multiply_dense(Ho, 2.0, X)) < TOL


def test_empty_and_errors(ctx):
    fx = load("weak")
    H = build(D, fx, ctx)
    out = H.Multiply(1.0, np.zeros((H.Width(), 0)))
    assert out.shape == (H.Height(), 0)
    with pytest.raises(D.HMError):
        H.Multiply(1.0, np.zeros(H.Width() + 1))
