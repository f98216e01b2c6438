"""The MLP oracle's analytic gradient against central finite differences (float64)."""
import numpy as np

from oracle import mlp_oracle as M


def test_oracle_gradient_is_the_derivative():
    rng = np.random.default_rng(0)
    in_dim, H = 12, 8
    n = H * in_dim + H + H * H + H + H + 1
    w = rng.normal(0, 0.5, n)
    x = rng.normal(0, 1, (6, in_dim))
    t = rng.normal(0, 1, 6)
    _, _, g = M.forward_backward(w, x, t, in_dim, H, round_weights=False)
    eps = 1e-6
    num = np.empty(n)
    for i in range(n):
        wp, wm = w.copy(), w.copy()
        wp[i] += eps
        wm[i] -= eps
        num[i] = (M.forward_backward(wp, x, t, in_dim, H, False)[1] - M.forward_backward(wm, x, t, in_dim, H, False)[1]) / (2 * eps)
    np.testing.assert_allclose(g, num, rtol=1e-5, atol=1e-8)


def test_bf16_rounding_is_nearest_even():
    v = np.array([1.0, 1.00390625, 1.005859375, -3.1415927, 65504.0], np.float32)
    r = M.bf16_round(v)
    # bf16 keeps 8 significant bits: spacing 2^-7 around 1
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125
    assert abs(r[3] + 3.140625) < 1e-12
