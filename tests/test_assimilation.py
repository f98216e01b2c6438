"""Ensemble Kalman filter restatement against the reference's diffusion_enkf
(golden fixture made by tests/golden/make_golden.py --enkf)."""
import os

import numpy as np
import pytest
import torch

from digital_twin_brain_b200.assimilation import diffusion_enkf, log_torch, sigmoid_torch
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
