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


SKETCH = 8


def hashed_uniform(n, k, seed):
    """n x k matrix (column-major element order i + j n) of uniforms in
    [-1, 1) from the splitmix64 hash of (seed, element index); exact on every
    machine and numpy version."""
    with np.errstate(over="ignore"):
        z = (np.arange(n * k, dtype=np.uint64)
             + np.uint64(seed) * np.uint64(0xD1B54A32D192ED03)
             + np.uint64(0x9E3779B97F4A7C15))
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    u = (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return (2.0 * u - 1.0).reshape(k, n).T.copy()


def big_case_inputs(spec):
    """Coefficient field (natural order), right-hand sides and sketch matrix
    of a benchmark-size case (a make_golden.BIG_CASES entry, or the fixture
    it wrote: keys sizes, seed, nrhs and coef / coef_kind = "uniform" for c in
    [1, 2) or "log_uniform" for c in [1, 100))."""
    N = int(np.prod(spec["sizes"]))
    s = int(spec["seed"])
    kind = str(spec["coef_kind"] if "coef_kind" in spec else spec["coef"])
    u = 0.5 * (hashed_uniform(N, 1, s)[:, 0] + 1.0)               # [0, 1)
    coef = 1.0 + u if kind == "uniform" else 100.0 ** u
    X = hashed_uniform(N, int(spec["nrhs"]), s + 1)
    G = hashed_uniform(N, SKETCH, s + 2)
    return coef, X, G
