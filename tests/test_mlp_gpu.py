"""The rank predictor's GPU kernels: forward and gradient against the CPU
oracle (oracle/mlp_oracle.py; FP32 on the GPU, so 1e-4 relative), training
lowers the loss, and the learned sample counts in H*H: fewer samples than
the fixed count, the probe check redoing the compressions it rejects, and
the product still at the tolerance's accuracy."""
import numpy as np
import pytest

import dmhm_b200 as D
from helpers import build, load, relerr
from oracle import mlp_oracle as M

pytestmark = pytest.mark.gpu


def test_forward_and_gradient_match_oracle():
    ctx = D.Context(0)
    m = D.RankModel(ctx, seed=3)
    rng = np.random.default_rng(1)
    x = rng.random((300, M.F)).astype(np.float32)
    t = rng.random(300).astype(np.float32)
    p = m.params().astype(np.float64)
    y_ref, _ = M.forward(p, x)
    assert np.max(np.abs(m.predict(x) - y_ref)) < 1e-5
    loss, g = m.loss_grad(x, t)
    loss_ref, g_ref = M.loss_grad(p, x, t)
    assert abs(loss - loss_ref) <= 1e-5 * max(1.0, loss_ref)
    assert np.linalg.norm(g - g_ref) <= 1e-4 * np.linalg.norm(g_ref)


def test_training_lowers_loss_deterministically():
    ctx = D.Context(0)
    rng = np.random.default_rng(2)
    x = rng.random((500, M.F)).astype(np.float32)
    t = (0.2 + 0.6 * x[:, 0] * x[:, 3]).astype(np.float32)
    m1, m2 = D.RankModel(ctx, seed=5), D.RankModel(ctx, seed=5)
    l0, _ = m1.loss_grad(x, t)
    l1 = m1.train(x, t, epochs=300, lr=1e-2)
    l2 = m2.train(x, t, epochs=300, lr=1e-2)
    assert l1 < 0.2 * l0
    assert l1 == l2 and np.array_equal(m1.params(), m2.params())


def _schulz_iterate(fx, ctx, its=4):
    X = build(D, fx, ctx)
    X.SchulzInvert(its, 1.5, 6.0, 1e-30)
    return X


def _log_and_train(fx, tol, epochs=400):
    ctx = D.Context(0)
    ctx.set_oversample(int(fx["oversample"]))
    ctx.set_compression_tolerance(tol)
    ctx.rank_log_enable(True)
    _schulz_iterate(fx, ctx, 5)
    x, t = ctx.rank_log(clear=True)
    ctx.rank_log_enable(False)
    m = D.RankModel(ctx, seed=7)
    m.train(x, t, epochs=epochs, lr=1e-2)
    return ctx, m, x, t


def _products(fx, ctx, model, margin):
    """X A with the fixed sample count, then with the model attached."""
    X = _schulz_iterate(fx, ctx, 3)
    A = build(D, fx, ctx)
    s0 = ctx.rank_stats()
    C_plain = X.Multiply(1.0, A)
    s1 = ctx.rank_stats()
    ctx.use_rank_model(model, margin=margin, probes=4)
    C_learn = X.Multiply(1.0, A)
    s2 = ctx.rank_stats()
    ctx.use_rank_model(None)
    d1 = {k: s1[k] - s0[k] for k in s0}
    d2 = {k: s2[k] - s1[k] for k in s0}
    return C_plain, C_learn, d1, d2


def test_learned_sample_counts_save_samples_and_keep_accuracy():
    fx = load("c1")
    ctx, model, x, t = _log_and_train(fx, 1e-8)
    assert x.shape[0] > 0 and np.all((t >= 0) & (t <= 1))
    C_plain, C_learn, d_plain, d_learn = _products(fx, ctx, model, margin=2)
    assert d_learn["samples"] < d_plain["samples"]
    P = fx["probes"]
    assert relerr(C_learn.Multiply(1.0, P), C_plain.Multiply(1.0, P)) < 1e-6


def test_probe_check_redoes_underestimated_blocks():
    """A model that predicts rank 0 everywhere must be caught by the probe
    check: the compressions with content are redone and the product matches
    the fixed-count one."""
    fx = load("c1")
    ctx = D.Context(0)
    ctx.set_oversample(int(fx["oversample"]))
    ctx.set_compression_tolerance(1e-8)
    m = D.RankModel(ctx, seed=1)
    p = np.zeros(D.RankModel.num_params(), dtype=np.float32)
    p[-1] = -30.0   # output bias: sigmoid ~ 0
    m.set_params(p)
    C_plain, C_learn, _, d_learn = _products(fx, ctx, m, margin=0)
    assert d_learn["fallbacks"] > 0
    P = fx["probes"]
    assert relerr(C_learn.Multiply(1.0, P), C_plain.Multiply(1.0, P)) < 1e-6
