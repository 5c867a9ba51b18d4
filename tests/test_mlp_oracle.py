"""The network oracle's own backward, pinned by finite differences (CPU)."""
import numpy as np

from oracle import mlp_oracle as mo


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.0, 0.0], dtype=np.float32)
    r = mo.bf16(x)
    assert r[0] == 1.0 and r[3] == -3.0 and r[4] == 0.0
    assert r[1] == 1.0            # halfway, rounds to even
    assert r[2] == 1.0078125      # above halfway, rounds up


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(3)
    p = mo.init(5, scale=0.5).astype(np.float64)
    x = rng.uniform(-1, 1, (16, mo.F))
    t = rng.uniform(-1, 1, 16)
    loss, g = mo.grads(p, x, t, exact=True)
    idx = np.concatenate([rng.integers(mo.OFF_W1, mo.OFF_B1, 6), rng.integers(mo.OFF_B1, mo.OFF_W2, 4),
                          rng.integers(mo.OFF_W2, mo.OFF_B2, 8), rng.integers(mo.OFF_B2, mo.OFF_W3, 4),
                          rng.integers(mo.OFF_W3, mo.OFF_B3, 4), [mo.OFF_B3]])
    h = 1e-6
    for i in idx:
        q = p.copy()
        q[i] += h
        lp = mo.grads(q, x, t, exact=True)[0]
        q[i] -= 2 * h
        lm = mo.grads(q, x, t, exact=True)[0]
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(fd)), (i, fd, g[i])


def test_level_stats_small():
    import oracle
    # path 0-1-2-3 as a 2-regular cycle of 4 (square): distances 1,1,2
    adj = np.array([[1, 3], [0, 2], [1, 3], [2, 0]])
    st = oracle.level_stats(adj, 4)
    assert st[:, 0].tolist() == [3] * 4
    assert st[:, 1].tolist() == [1] * 4
    assert st[:, 2].tolist() == [0] * 4
