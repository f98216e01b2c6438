"""Ensemble Kalman filter restatement against the reference's diffusion_enkf
(golden fixture made by tests/golden/make_golden.py --enkf)."""
import os

import numpy as np
import pytest
import torch

from digital_twin_brain_b200.assimilation import diffusion_enkf, judge_error, log_torch, sigmoid_torch
from digital_twin_brain_b200.surrogate import HISTORY, with_context
from tests._helpers import GOLDEN


@pytest.mark.parametrize("case", ["small", "da"])
def test_diffusion_enkf_matches_reference(case):
    g = np.load(os.path.join(GOLDEN, "enkf_ref.npz"))
    w = diffusion_enkf(torch.from_numpy(g[f"{case}_w_hat"]), float(g["bold_sigma"]),
                       torch.from_numpy(g[f"{case}_bold_t"]), float(g["solo_rate"]),
                       noise=torch.from_numpy(g[f"{case}_noise"]))
    np.testing.assert_allclose(w.numpy(), g[f"{case}_w"], rtol=1e-6, atol=1e-6)


def test_bounded_transform_roundtrip():
    lo = torch.full((4,), 0.5)
    hi = torch.full((4,), 1.5)
    x = torch.linspace(-30, 30, 40).reshape(10, 4)
    y = sigmoid_torch(x, lo, hi)
    assert (y > lo).all() and (y < hi).all()
    np.testing.assert_allclose(log_torch(y, lo, hi).numpy(), x.numpy(), rtol=1e-3, atol=1e-3)


def test_judge_error_is_absolute_error_relative_to_the_total_rate():
    r = torch.tensor([[0.01, 0.02], [0.03, 0.04]])
    assert judge_error(r, r) == 0.0
    e = judge_error(r * 1.1, r)
    assert abs(e - 0.1 * 0.1 / (0.1 + 4e-5)) < 1e-6
    assert abs(judge_error(r * 11.0, r * 10.0) - e) < 1e-3           # nearly scale-free
    quiet = torch.tensor([[1e-4, 0.05]])                               # a near-silent region off by 3x
    assert judge_error(torch.tensor([[3e-4, 0.05]]), quiet) < 0.005


def test_surrogate_inputs_carry_the_member_mean_of_the_last_windows():
    M, R = 3, 5
    hist = torch.arange(M * R * HISTORY, dtype=torch.float32).reshape(M, R, HISTORY)
    x = with_context(hist, 2)
    assert x.shape == (M * R, HISTORY + 2)
    assert torch.equal(x[:, :HISTORY], hist.reshape(-1, HISTORY))
    for m in range(M):
        ctx = hist[m, :, HISTORY - 2:].mean(0)
        for r in range(R):
            assert torch.equal(x[m * R + r, HISTORY:], ctx)
    assert torch.equal(with_context(hist, 0), hist.reshape(-1, HISTORY))

