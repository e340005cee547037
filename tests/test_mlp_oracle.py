"""The float64 network oracle itself: without the BF16 roundings its gradient
equals central finite differences of its loss."""

from __future__ import annotations

import numpy as np

from oracle import mlp as M


def test_oracle_gradient_matches_finite_differences(monkeypatch):
    monkeypatch.setattr(M, "bf16", lambda x: np.asarray(x, dtype=np.float64))
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.3, M.N_PARAMS)
    x = rng.normal(size=(37, 8))
    t = rng.normal(size=37)
    _, g = M.loss_and_grad(p, x, t)
    idx = rng.choice(M.N_PARAMS, 60, replace=False)
    idx = np.concatenate([idx, [M.OFF_B3, M.OFF_W3 + 5, M.OFF_B1 + 7, M.OFF_W1 + 3]])
    eps = 1e-6
    for i in idx:
        q = p.copy()
        q[i] += eps
        lp, _ = M.loss_and_grad(q, x, t)
        q[i] -= 2 * eps
        lm, _ = M.loss_and_grad(q, x, t)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])


def test_bf16_rounding_is_nearest_even():
    vals = np.array([1.0, 1.00390625, 1.005859375, -2.5, 3.0e-3], dtype=np.float32)
    r = M.bf16(vals)
    assert r[0] == 1.0 and r[1] == 1.0            # halfway, rounds to even
    assert r[2] == 1.0078125                       # above halfway, rounds up
    assert r[3] == -2.5
    assert abs(r[4] - 3.0e-3) / 3.0e-3 < 2 ** -8
