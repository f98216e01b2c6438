"""Input neurons (models/block.py:37-50, :104-109) on the device against the
reference's own run of the same network (golden fixture)."""
import os

import numpy as np
import pytest
import torch

from digital_twin_brain_b200.models.block import block
from digital_twin_brain_b200 import Network
from digital_twin_brain_b200._lib import DtbError
from tests._helpers import GOLDEN, unpack

pytestmark = pytest.mark.gpu


def _w(g):
    post, pre, kind, w = g["post"], g["pre"], g["kind"], g["w"]
    N = g["prop"].shape[0]
    idx = np.stack([kind.astype(np.int64), post.astype(np.int64), pre.astype(np.int64)])
    idx = np.stack([idx, idx], axis=-1)
    idx[0, :, 1] += 1
    return torch.sparse_coo_tensor(torch.from_numpy(idx.reshape(3, -1)), torch.from_numpy(w.reshape(-1).copy()),
                                   (4, N, N))


@pytest.mark.parametrize("stepwise", [True, False])
def test_input_neurons_bit_exact_vs_reference(stepwise):
    g = np.load(os.path.join(GOLDEN, "src_block_ref.npz"))
    N = g["prop"].shape[0]
    b = block(torch.from_numpy(g["prop"]), _w(g), delta_t=float(g["dt"]), src=torch.from_numpy(g["src"]),
              seed=int(g["seed"]), device=0)
    assert np.array_equal(b.src_neuron.numpy(), np.arange(g["src"].shape[0]))
    act = unpack(g["active"], N)
    steps = int(g["steps"])
    if stepwise:
        for k in range(steps):
            s, m = b.run(noise_rate=0.01)
            assert np.array_equal(b.active.numpy(), act[k]), k
            assert np.array_equal(b.V_i.numpy(), g["V"][k]), k
            assert np.array_equal(s.numpy(), g["sums"][k])
    else:
        s, m = b.run_steps(steps, noise_rate=0.01)
        assert np.array_equal(s.numpy(), g["sums"])
        assert np.array_equal(b.V_i.numpy(), g["V"][-1])
    assert np.array_equal(b.J_ui.numpy(), g["J_final"])
    assert np.array_equal(b.I_syn.numpy(), g["I_syn_final"])
    assert np.array_equal(b.t_ik_last.numpy(), g["t_last_final"])
    with pytest.raises(IndexError):       # the reference raises on the step past its raster
        b.run(noise_rate=0.01)
    with pytest.raises(DtbError):         # and so does the C ABI
        b.network.run(1, 0.01)


def test_input_neurons_replaced_and_removed():
    g = np.load(os.path.join(GOLDEN, "src_block_ref.npz"))
    b = block(torch.from_numpy(g["prop"]), _w(g), delta_t=float(g["dt"]), src=torch.from_numpy(g["src"]),
              seed=int(g["seed"]), device=0)
    net = b.network
    n_src = g["src"].shape[0]
    before = net.info().device_bytes
    net.set_input_spikes(np.arange(n_src), g["src"])        # replaced: same footprint afterwards
    assert net.info().device_bytes == before
    net.run(10, 0.01)
    net.set_input_spikes([], None)                            # removed: the network runs free
    net.run(500, 0.01)
