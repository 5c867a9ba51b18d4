"""The proposal filter's network on the GPU against its CPU oracle.

Tolerance: the device accumulates in FP32 and the oracle in float64 with the
same BF16 rounding points, so values agree to about 1e-3 relative; a rounding
boundary crossed differently moves single BF16 activations by one unit in the
last place.  Forward outputs must agree within 2% of their range and every
gradient block within 2% in relative L2 norm -- a wrong fragment layout or
transpose gives errors of order 100%."""
import numpy as np
import pytest

import graphgolf_b200 as gg
from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu

BLOCKS = {"W1": (mo.OFF_W1, mo.OFF_B1), "b1": (mo.OFF_B1, mo.OFF_W2), "W2": (mo.OFF_W2, mo.OFF_B2),
          "b2": (mo.OFF_B2, mo.OFF_W3), "w3": (mo.OFF_W3, mo.OFF_B3), "b3": (mo.OFF_B3, mo.N_PARAMS)}


@pytest.fixture(scope="module")
def net(gpu):
    n = gg.FilterNet(max_rows=4096, seed=1)
    yield n
    n.close()


def test_param_roundtrip(net):
    p = mo.init(11)
    net.params = p
    assert np.array_equal(net.params, p)


@pytest.mark.parametrize("rows", [16, 64, 4096])
def test_forward_matches_oracle(net, rows):
    rng = np.random.default_rng(rows)
    p = mo.init(7)
    net.params = p
    x = rng.uniform(-1, 1, (rows, 32)).astype(np.float32)
    y = net.forward(x)
    y_ref, _ = mo.forward(p, x)
    assert np.abs(y - y_ref).max() <= 0.02 * (np.abs(y_ref).max() + 1e-6)


@pytest.mark.parametrize("rows", [16, 64, 256])
def test_gradients_match_oracle(net, rows):
    rng = np.random.default_rng(100 + rows)
    p = mo.init(9)
    net.params = p
    x = rng.uniform(-1, 1, (rows, 32)).astype(np.float32)
    t = rng.uniform(-2, 2, rows).astype(np.float32)
    loss, g = net.grads(x, t)
    loss_ref, g_ref = mo.grads(p, x, t)
    assert abs(loss - loss_ref) <= 0.02 * loss_ref
    for name, (a, b) in BLOCKS.items():
        err = np.linalg.norm(g[a:b] - g_ref[a:b]) / (np.linalg.norm(g_ref[a:b]) + 1e-12)
        assert err < 0.02, (name, err)


def test_adam_first_step(net):
    """Adam's first step moves every parameter by lr * g / (|g| + eps)."""
    rng = np.random.default_rng(5)
    p = mo.init(13)
    net.params = p
    net.set_adam(lr=1e-3)
    x = rng.uniform(-1, 1, (64, 32)).astype(np.float32)
    t = rng.uniform(-1, 1, 64).astype(np.float32)
    _, g = net.grads(x, t)
    net.params = p          # resets Adam
    net.train(x, t, 1)
    step = p - net.params
    big = np.abs(g) > 1e-4 * np.abs(g).max()
    want = 1e-3 * g[big] / (np.abs(g[big]) + 1e-8)
    assert np.allclose(step[big], want, rtol=1e-3, atol=1e-7)


def test_training_fits(net):
    rng = np.random.default_rng(21)
    net.params = mo.init(1, scale=0.5)
    net.set_adam(lr=1e-3)
    x = rng.uniform(-1, 1, (256, 32)).astype(np.float32)
    t = (np.sin(2 * x[:, 0]) + x[:, 1] * x[:, 2] - 0.5 * x[:, 3]).astype(np.float32)
    first = net.grads(x, t)[0]
    last = net.train(x, t, 400)
    assert last < 0.1 * first


@pytest.mark.parametrize("rows", [208, 4000])
def test_forward_partial_tiles(net, rows):
    """Row counts that leave the last 128-row tile of the inference forward
    part-filled: every row is written and equals the oracle."""
    rng = np.random.default_rng(rows)
    p = mo.init(17)
    net.params = p
    x = rng.uniform(-1, 1, (rows, 32)).astype(np.float32)
    y = net.forward(x)
    y_ref, _ = mo.forward(p, x)
    assert np.isfinite(y).all()
    assert np.abs(y - y_ref).max() <= 0.02 * (np.abs(y_ref).max() + 1e-6)


def test_forward_after_adam(net):
    """Adam refreshes every BF16 copy the forwards read (row-major and the
    tensor cores' operand layout): after training, the forward equals the
    oracle's forward with the trained parameters."""
    rng = np.random.default_rng(31)
    net.params = mo.init(3, scale=0.5)
    net.set_adam(lr=3e-3)
    x = rng.uniform(-1, 1, (128, 32)).astype(np.float32)
    t = rng.uniform(-1, 1, 128).astype(np.float32)
    net.train(x, t, 20)
    p = net.params
    xs = rng.uniform(-1, 1, (512, 32)).astype(np.float32)
    y = net.forward(xs)
    y_ref, _ = mo.forward(p, xs)
    assert np.abs(y - y_ref).max() <= 0.02 * (np.abs(y_ref).max() + 1e-6)


def test_forward_timing(net):
    net.params = mo.init(5)
    x = np.random.default_rng(2).uniform(-1, 1, (4096, 32)).astype(np.float32)
    ms = net.time_forward(x, 20)
    assert 0.0 < ms < 5.0
