"""The cost model's CUDA kernels against the CPU backprop, and training
properties (GPU)."""
import numpy as np
import pytest

import mlp_ref
from ots import model


@pytest.mark.gpu
def test_cuda_forward_backward_match_cpu_backprop():
    rng = np.random.default_rng(3)
    n_in, hidden, layers = len(model.FEATURES), 32, 3
    m = model.MLP(n_in, hidden, layers, seed=11)
    X = rng.normal(0, 2, (300, n_in)).astype(np.float32)
    y = rng.normal(3, 1, 300).astype(np.float32)
    mean = X.mean(0)
    inv = 1.0 / X.std(0)
    m.set_normalization(mean, inv, 3.0, 1.0)
    loss, g = m.loss_grad(X, y)
    dims = mlp_ref.layer_dims(n_in, hidden, layers)
    rl, rg = mlp_ref.loss_grad(X, y, m.params().astype(np.float64), dims,
                               mean.astype(np.float64), inv.astype(np.float64), 3.0, 1.0)
    assert abs(loss - rl) <= 1e-5 * max(1.0, rl)
    err = np.max(np.abs(g - rg)) / max(1e-3, np.max(np.abs(rg)))
    assert err < 1e-4, err
    p = m.predict(X[:17])
    rp, _, _ = mlp_ref.forward(X[:17], m.params().astype(np.float64), dims, mean, inv)
    assert np.allclose(p, rp + 3.0, rtol=1e-5, atol=1e-5)


@pytest.mark.gpu
def test_training_is_deterministic_and_learns():
    rng = np.random.default_rng(4)
    X = rng.normal(0, 1, (512, 8)).astype(np.float32)
    y = (np.sin(X[:, 0]) + X[:, 1] * X[:, 2]).astype(np.float32)
    outs = []
    for _ in range(2):
        m = model.MLP(8, 32, 3, seed=5)
        m.fit_normalization(X, y)
        l0, _ = m.loss_grad(X, y)
        l1 = m.fit(X, y, epochs=150, batch=64, lr=3e-3, seed=9)
        outs.append(m.params())
        lf, _ = m.loss_grad(X, y)
        assert lf < 0.2 * l0, (l0, lf, l1)
    assert np.array_equal(outs[0], outs[1])


@pytest.mark.gpu
def test_topk_orders_predictions():
    rng = np.random.default_rng(6)
    m = model.MLP(4, 8, 2, seed=1)
    X = rng.normal(0, 1, (50, 4)).astype(np.float32)
    m.set_normalization(np.zeros(4), np.ones(4), 0.0, 1.0)
    p = m.predict(X)
    top = m.topk(X, 5)
    assert list(top) == list(np.argsort(-p, kind="stable")[:5])


@pytest.mark.gpu
@pytest.mark.parametrize("held", ["rician-denoise-2d", "cdsc-tv-update-2d"])
def test_learned_picker_finds_near_best_at_tenth_of_the_sweep(held):
    """Held-out stencils (trained on every other stencil's B200 sweep): the
    model's top 10 % contains a configuration within 5 % of the exhaustive
    best, and does at least as well as 10 % random picks (the method without
    the model at the same measuring cost)."""
    import json
    import os
    data = os.path.join(os.path.dirname(model.__file__), "data", "sweeps_b200.json")
    recs = json.load(open(data))["records"]
    rep = model.leave_one_out(recs, held_out=[held], epochs=300)
    r = rep[held]
    assert r["measure_cost"] <= 0.10
    assert r["picked_over_best"] >= 0.95
    assert r["picked_over_best"] >= r["random_k_over_best"]
