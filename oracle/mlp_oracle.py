"""CPU oracle (test infrastructure only) of the learned rank predictor's
perceptron: forward, mean-squared-error loss on the sigmoid output, and the
analytic gradient, in the parameter layout of the library's kernels
(dmhm_b200/csrc/mlp.cu).  The reference has no counterpart (its randomized
product always draws maxRank + Oversample() samples,
include/dmhm/hmat_tools.hpp:1657-1746); this restatement is checked against
central finite differences in tests/test_mlp.py and checks the GPU
gradients in tests/test_mlp_gpu.py.  Computed in float64."""
import numpy as np

F, H = 12, 64
OW1, OB1 = 0, H * F
OW2, OB2 = OB1 + H, OB1 + H + H * H
OW3, OB3 = OB2 + H, OB2 + H + H
NPARAM = OB3 + 1


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[OW1:OB1].reshape(H, F), p[OB1:OW2], p[OW2:OB2].reshape(H, H), p[OB2:OW3],
            p[OW3:OB3], p[OB3])


def forward(p, x):
    W1, b1, W2, b2, w3, b3 = unpack(p)
    x = np.asarray(x, dtype=np.float64)
    z1 = x @ W1.T + b1
    a1 = np.maximum(z1, 0.0)
    z2 = a1 @ W2.T + b2
    a2 = np.maximum(z2, 0.0)
    z3 = a2 @ w3 + b3
    y = 1.0 / (1.0 + np.exp(-z3))
    return y, (x, z1, a1, z2, a2, z3)


def loss(p, x, t):
    y, _ = forward(p, x)
    return float(np.mean((y - np.asarray(t, dtype=np.float64)) ** 2))


def loss_grad(p, x, t):
    W1, b1, W2, b2, w3, b3 = unpack(p)
    y, (x, z1, a1, z2, a2, z3) = forward(p, x)
    t = np.asarray(t, dtype=np.float64)
    n = y.size
    dz3 = 2.0 * (y - t) * y * (1.0 - y) / n
    g = np.zeros(NPARAM)
    g[OW3:OB3] = a2.T @ dz3
    g[OB3] = dz3.sum()
    dz2 = np.outer(dz3, w3) * (z2 > 0)
    g[OW2:OB2] = (dz2.T @ a1).ravel()
    g[OB2:OW3] = dz2.sum(axis=0)
    dz1 = (dz2 @ W2) * (z1 > 0)
    g[OW1:OB1] = (dz1.T @ x).ravel()
    g[OB1:OW2] = dz1.sum(axis=0)
    return float(np.mean((y - t) ** 2)), g
