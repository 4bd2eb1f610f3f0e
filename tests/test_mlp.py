"""The CPU restatement of the rank predictor's perceptron (oracle/
mlp_oracle.py): its analytic gradient against central finite differences,
and the library's parameter/feature counts (no GPU needed)."""
import numpy as np

from oracle import mlp_oracle as M


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.standard_normal(M.NPARAM) * 0.3
    x = rng.random((40, M.F))
    t = rng.random(40)
    _, g = M.loss_grad(p, x, t)
    h = 1e-6
    idx = rng.choice(M.NPARAM, 60, replace=False)
    for i in idx:
        e = np.zeros(M.NPARAM)
        e[i] = h
        fd = (M.loss(p + e, x, t) - M.loss(p - e, x, t)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd))


def test_layout_matches_library():
    import dmhm_b200 as D
    assert D.RankModel.num_features() == M.F
    assert D.RankModel.num_params() == M.NPARAM
