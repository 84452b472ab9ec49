"""The CPU restatement of the indicator network: its back-propagation
against finite differences (float64, no rounding)."""
import numpy as np

import mlp_oracle as M


def test_backprop_matches_finite_differences():
    rng = np.random.default_rng(1)
    P = M.init_params(3)
    X = rng.normal(0, 0.6, (64, M.NIN))
    y = (rng.uniform(size=64) < 0.3).astype(np.float64)
    G, _ = M.grads_exact(P, X, y, pos_weight=2.5)
    idx = np.concatenate([rng.choice(M.NPARAM, 40, replace=False), [M.OFF_B3, M.OFF_B1 + 3, M.OFF_W3 + 7]])
    h = 1e-6
    for i in idx:
        Pp, Pm = P.copy(), P.copy()
        Pp[i] += h
        Pm[i] -= h
        fd = (M.loss_exact(Pp, X, y, 2.5) - M.loss_exact(Pm, X, y, 2.5)) / (2 * h)
        assert abs(fd - G[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, G[i])


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -7, 1.0 + 3 * 2 ** -8, -3.3])
    r = M.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -7 and r[3] == 1.0 + 2 ** -6
    assert abs(r[4] + 3.3) < 2 ** -6
