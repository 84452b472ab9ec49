"""The tensor-core (tcgen05) kernels of the indicator network against the
CPU restatement with the same BF16 rounding points: forward logits and
parameter gradients; and training drives the loss down."""
import numpy as np
import pytest

import mlp_oracle as M

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def MLP():
    from finess_b200.indicator import MLP as cls
    return cls


def test_forward_matches_emulated_oracle(MLP):
    rng = np.random.default_rng(0)
    P = M.init_params(1)
    X = rng.normal(0, 0.7, (1000, M.NIN)).astype(np.float32)   # ragged: 7 full tiles + 104 rows
    m = MLP(params=P.astype(np.float32))
    z = m.forward(X)
    zo = M.forward_emulated(P.astype(np.float32).astype(np.float64), X.astype(np.float64))
    assert np.max(np.abs(z - zo)) <= 2e-3 * max(1.0, np.max(np.abs(zo)))


def test_gradients_match_emulated_oracle(MLP):
    rng = np.random.default_rng(2)
    P = M.init_params(4).astype(np.float32).astype(np.float64)
    X = rng.normal(0, 0.7, (300, M.NIN)).astype(np.float32)
    y = (rng.uniform(size=300) < 0.4).astype(np.uint8)
    m = MLP(params=P.astype(np.float32))
    g, loss = m.gradients(X, y, pos_weight=3.0)
    go, lo = M.grads_emulated(P, X.astype(np.float64), y, 3.0)
    assert abs(loss - lo) <= 1e-3 * abs(lo)
    for a, b in ((M.OFF_W1, M.OFF_B1), (M.OFF_B1, M.OFF_W2), (M.OFF_W2, M.OFF_B2), (M.OFF_B2, M.OFF_W3),
                 (M.OFF_W3, M.OFF_B3), (M.OFF_B3, M.NPARAM)):
        scale = max(np.max(np.abs(go[a:b])), 1e-6)
        assert np.max(np.abs(g[a:b] - go[a:b])) <= 2e-2 * scale, (a, b)


def test_training_reduces_loss(MLP):
    rng = np.random.default_rng(5)
    X = rng.normal(0, 1.0, (20000, M.NIN)).astype(np.float32)
    y = (X[:, 0] + 0.5 * X[:, 3] - 0.2 * X[:, 7] > 0.3).astype(np.uint8)
    m = MLP(seed=11)
    losses = m.train(X, y, epochs=6, batch=2048, lr=3e-3)
    assert losses[-1] < 0.6 * losses[0], losses
    acc = np.mean((m.forward(X) > 0) == (y > 0))
    assert acc > 0.9, acc
