"""Surrogate MLP kernels: forward and gradients against the float64 CPU oracle,
and training that fits a smooth function."""
import numpy as np
import pytest
import torch

from oracle import mlp_oracle
from digital_twin_brain_b200.surrogate import MLP, RateSurrogate

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("B", [1, 37, 3000])
def test_forward_and_gradient_match_oracle(B):
    rng = np.random.default_rng(B)
    m = MLP(12, 256, seed=3, device=0)
    x = rng.normal(0, 1, (B, 12)).astype(np.float32)
    t = rng.normal(0, 1, B).astype(np.float32)
    w = m.params()
    y_ref, loss_ref, g_ref = mlp_oracle.forward_backward(w, x, t, 12, 256)
    y = m.forward(torch.from_numpy(x)).cpu().numpy()
    np.testing.assert_allclose(y, y_ref, rtol=1e-4, atol=1e-5)
    g, loss = m.gradient(torch.from_numpy(x), torch.from_numpy(t))
    g = g.cpu().numpy()
    assert abs(loss - loss_ref) <= 1e-4 * max(loss_ref, 1e-6)
    scale = np.abs(g_ref).max()
    assert np.abs(g - g_ref).max() <= 1e-4 * scale, np.abs(g - g_ref).max() / scale


def test_training_fits_a_function():
    rng = np.random.default_rng(0)
    x = rng.uniform(-2, 2, (20000, 12)).astype(np.float32)
    t = (np.sin(x[:, 0]) + 0.5 * x[:, 1] * x[:, 2] - 0.3 * x[:, 3]).astype(np.float32)
    m = MLP(12, 256, seed=1, device=0)
    hist = m.fit(torch.from_numpy(x), torch.from_numpy(t), epochs=40, batch=1024, lr=2e-3)
    assert hist[-1] < 0.05 * hist[0] and hist[-1] < 0.02


def test_rate_surrogate_learns_rate_map():
    """A synthetic rate law (rate depends on g factors and the last window) is learned
    well enough to beat the persistence forecast (the method without the network)."""
    rng = np.random.default_rng(1)
    n = 30000
    gui = rng.uniform(0.5, 1.5, (n, 4)).astype(np.float32)
    hist = rng.uniform(0.0005, 0.01, (n, 8)).astype(np.float32)
    target = (0.6 * hist[:, -1] * gui[:, 0] / gui[:, 2] + 0.002 * gui[:, 1]).astype(np.float32)
    s = RateSurrogate(seed=2, context=0)
    s.fit(torch.from_numpy(gui), torch.from_numpy(hist), torch.from_numpy(target), epochs=40, lr=2e-3)
    pred = s.predict(torch.from_numpy(gui), torch.from_numpy(hist)).cpu().numpy()
    err_net = np.sqrt(np.mean((pred - target) ** 2))
    err_persist = np.sqrt(np.mean((hist[:, -1] - target) ** 2))
    assert err_net < 0.25 * err_persist, (err_net, err_persist)
