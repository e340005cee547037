"""Float64 restatement of the step-size network's forward and backward pass.

TEST INFRASTRUCTURE ONLY: the checker of the package's training and
inference kernels.  The network is 8 -> 64 -> 64 -> 1 with SiLU, BF16 weights
and BF16 inputs / hidden activations (round to nearest even), FP32 biases,
loss = mean squared error; SiLU(z) = z (1 + tanh(z/2)) / 2 with the tanh
argument and result rounded to BF16 like the kernels' tanh.approx.bf16x2.
Gradients pass straight through the roundings.
"""

from __future__ import annotations

import numpy as np

OFF_W1, OFF_B1, OFF_W2, OFF_B2, OFF_W3, OFF_B3, N_PARAMS = 0, 512, 576, 4672, 4736, 4800, 4801


def bf16(x) -> np.ndarray:
    """Round float32 values to the nearest bfloat16 (ties to even), as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p: np.ndarray):
    p = np.asarray(p, dtype=np.float64)
    return (p[OFF_W1:OFF_B1].reshape(8, 64), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(64, 64), p[OFF_B2:OFF_W3],
            p[OFF_W3:OFF_B3], p[OFF_B3])


def _silu(z):
    t = bf16(np.tanh(bf16(0.5 * z)))
    s = 0.5 + 0.5 * t
    return z * s, s


def forward(p, x):
    """x: (n, 8) standardised features -> (n,) output and the intermediates."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    W1, W2, W3 = bf16(W1), bf16(W2), bf16(W3)
    xb = bf16(x)
    z1 = xb @ W1 + b1
    a1, s1 = _silu(z1)
    a1 = bf16(a1)
    z2 = a1 @ W2 + b2
    a2, s2 = _silu(z2)
    a2 = bf16(a2)
    y = a2 @ W3 + b3
    return y, (xb, z1, s1, a1, z2, s2, a2, W2, W3)


def loss_and_grad(p, x, t):
    """Mean squared error over the rows and its gradient (straight-through)."""
    y, (xb, z1, s1, a1, z2, s2, a2, W2, W3) = forward(p, x)
    n = x.shape[0]
    err = y - t
    dy = 2.0 * err / n
    g = np.zeros(N_PARAMS)
    g[OFF_W3:OFF_B3] = a2.T @ dy
    g[OFF_B3] = dy.sum()
    dz2 = (dy[:, None] * W3[None, :]) * (s2 + z2 * s2 * (1.0 - s2))
    g[OFF_W2:OFF_B2] = (a1.T @ dz2).ravel()
    g[OFF_B2:OFF_W3] = dz2.sum(axis=0)
    dz1 = (dz2 @ W2.T) * (s1 + z1 * s1 * (1.0 - s1))
    g[OFF_W1:OFF_B1] = (xb.T @ dz1).ravel()
    g[OFF_B1:OFF_W2] = dz1.sum(axis=0)
    return float(np.mean(err ** 2)), g
