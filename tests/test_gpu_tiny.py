"""Edge sizes on the device against the oracle: one neuron (with and without a
self-synapse), fewer neurons than one 128-neuron tile, ragged last tiles, and a
network without synapses."""
import numpy as np
import pytest

from oracle import oracle as O
from digital_twin_brain_b200 import Network, synthetic
from digital_twin_brain_b200._lib import FIELD_J, FIELD_V
from tests._helpers import decay_like_reference

pytestmark = pytest.mark.gpu


def tiny_network(N: int, K: int):
    spec = synthetic.single_block(N, K, name=f"tiny_{N}_{K}")
    prop = spec.property()
    rng = np.random.default_rng(N * 7 + K)
    post = np.repeat(np.arange(N), K).astype(np.uint32)
    pre = rng.integers(0, N, N * K).astype(np.uint32)
    kind = (rng.integers(0, 2, N * K) * 2).astype(np.uint8)
    w = rng.uniform(0.0, 1.0, (N * K, 2)).astype(np.float32)
    return spec, prop, post, pre, kind, w


@pytest.mark.parametrize("N, K", [(1, 0), (1, 1), (100, 0), (127, 4), (129, 6), (300, 2)])
def test_tiny_ragged_and_synapse_free_networks_match_oracle(N, K):
    spec, prop, post, pre, kind, w = tiny_network(N, K)
    dec = decay_like_reference(prop, spec.dt)
    net = Network.from_arrays(prop, post, pre, kind, w, spec.dt, seed=3, decay=np.ascontiguousarray(dec.T))
    rowptr, opre, okind, ow = O.pull_csr(N, post, pre, kind, w)
    ob = O.OracleBlock(prop, dec, rowptr, opre, okind, ow, spec.dt, 3)
    spikes = 0
    for rate in (0.05, 0.3):          # the ordered push and, above 10 % activity, the streamed gather
        for _ in range(60):
            s, _, _ = net.run(1, noise_rate=rate, mode="pull")
            so, _ = ob.run(rate)
            assert np.array_equal(s[0], so)
            spikes += int(so.sum())
        assert np.array_equal(net.get(FIELD_V), ob.V)
        assert np.array_equal(net.get(FIELD_J), ob.J)
    net.synchronize()
    assert spikes >= 0
