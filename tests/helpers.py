"""Shared test helpers: fixture loading and relative errors."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def relerr(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def build(D, fx, ctx, coef_key="coef"):
    """H-matrix of a fixture case through the engine's public API."""
    sizes = [int(s) for s in fx["sizes"]]
    L = int(fx["levels"])
    S = D.operators.stencil(sizes, fx[coef_key], L)
    cls = D.HMat2d if len(sizes) == 2 else D.HMat3d
    return cls(S, L, int(fx["rank"]), bool(fx["strong"]), *sizes, ctx=ctx)


def stencil_exact(fx):
    """Exact A*A P, -0.5 A*B P and inv(A) P for a fixture's stencil
    operators A (coef) and B (coefB) on its probes P, by dense algebra."""
    from dmhm_b200 import operators as ops
    sizes = [int(s) for s in fx["sizes"]]
    L = int(fx["levels"])
    A = ops.dense_from_sparse(ops.stencil(sizes, fx["coef"], L))
    B = ops.dense_from_sparse(ops.stencil(sizes, fx["coefB"], L))
    P = fx["probes"]
    return dict(AA=A @ (A @ P), AB=-0.5 * (A @ (B @ P)), inv=np.linalg.solve(A, P))
