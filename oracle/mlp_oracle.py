"""CPU oracle of the proposal filter's network (TEST INFRASTRUCTURE ONLY).

A numpy restatement of the network in graphgolf_b200/csrc/mlp.cu, with BF16
rounding at the same points: inputs, W1, W2, the first hidden layer after
bias and ReLU, and the two gradients that enter tensor-core products (dZ2,
dZ1).  Products are accumulated in float64 here (the device accumulates in
FP32, so comparisons use a tolerance).  The network has no counterpart in
the reference; parity here is with this restatement of its mathematics, and
the restatement's own backward is pinned by finite differences in float64
(``exact=True`` turns every rounding off).

Packed parameters: W1 [256][32], b1 [256], W2 [256][256] (row n = weights
into unit n), b2 [256], w3 [256], b3 [1].
"""
from __future__ import annotations

import numpy as np

F, H = 32, 256
OFF_W1 = 0
OFF_B1 = OFF_W1 + H * F
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H
N_PARAMS = OFF_B3 + 1


def bf16(x) -> np.ndarray:
    """Round-to-nearest-even of float32 values to BF16, returned as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(a.shape)


def unpack(p):
    p = np.asarray(p)
    return (p[OFF_W1:OFF_B1].reshape(H, F), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(H, H), p[OFF_B2:OFF_W3],
            p[OFF_W3:OFF_B3], p[OFF_B3:])


def forward(p, x, exact: bool = False):
    """Returns (y, cache) for rows x [n][32]."""
    rnd = (lambda v: np.asarray(v, dtype=np.float64)) if exact else (lambda v: bf16(v).astype(np.float64))
    if not exact:
        p = np.asarray(p, dtype=np.float32)   # the device keeps FP32 master parameters
    W1, b1, W2, b2, w3, b3 = (np.asarray(a, dtype=np.float64) for a in unpack(p))
    X = rnd(x)
    W1r, W2r = rnd(W1), rnd(W2)
    Z1 = X @ W1r.T + b1
    H1 = rnd(np.maximum(Z1, 0.0))
    Z2 = H1 @ W2r.T + b2
    H2 = np.maximum(Z2, 0.0)
    y = H2 @ w3 + b3[0]
    return y, (X, W1r, W2r, H1, Z2, H2, w3)


def grads(p, x, t, exact: bool = False):
    """(loss, packed gradients) of mean((y - t)^2)."""
    rnd = (lambda v: np.asarray(v, dtype=np.float64)) if exact else (lambda v: bf16(v).astype(np.float64))
    y, (X, W1r, W2r, H1, Z2, H2, w3) = forward(p, x, exact)
    t = np.asarray(t, dtype=np.float64)
    B = X.shape[0]
    dy = 2.0 * (y - t) / B
    g = np.zeros(N_PARAMS, dtype=np.float64)
    g[OFF_W3:OFF_B3] = H2.T @ dy
    g[OFF_B3] = dy.sum()
    dz2 = (Z2 > 0) * dy[:, None] * w3[None, :]
    g[OFF_B2:OFF_W3] = dz2.sum(axis=0)
    dz2r = rnd(dz2)
    g[OFF_W2:OFF_B2] = (dz2r.T @ H1).ravel()
    dh1 = dz2r @ W2r
    dz1 = dh1 * (H1 > 0)
    g[OFF_B1:OFF_W2] = dz1.sum(axis=0)
    g[OFF_W1:OFF_B1] = (rnd(dz1).T @ X).ravel()
    return float(np.mean((y - t) ** 2)), g


def init(seed: int = 0, scale: float = 1.0) -> np.ndarray:
    """Seeded He-uniform parameters with small random biases (test input)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS, dtype=np.float32)
    p[OFF_W1:OFF_B1] = rng.uniform(-1, 1, H * F) * np.sqrt(6.0 / F) * scale
    p[OFF_B1:OFF_W2] = rng.uniform(-0.1, 0.1, H)
    p[OFF_W2:OFF_B2] = rng.uniform(-1, 1, H * H) * np.sqrt(6.0 / H) * scale
    p[OFF_B2:OFF_W3] = rng.uniform(-0.1, 0.1, H)
    p[OFF_W3:OFF_B3] = rng.uniform(-1, 1, H) * np.sqrt(6.0 / H)
    p[OFF_B3] = 0.05
    return p
