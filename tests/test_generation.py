"""Block files in the reference's layout (generation/make_block.py:473-479): what
generation.write_blocks writes reads back, through the restatement of
generation/read_block.py, as the same network with every postsynaptic row in the
order given."""
import os

import numpy as np

from digital_twin_brain_b200.generation import write_blocks
from tests._helpers import load_npz_blocks

KEYS = {"property": np.float32, "output_neuron_idx": np.uint32, "input_block_idx": np.int16,
        "input_neuron_idx": np.uint32, "input_channel_offset": np.uint8, "weight": np.float32}


def test_blocks_round_trip_keeps_rows_in_order(tmp_path):
    rng = np.random.default_rng(4)
    bounds = np.array([0, 70, 130, 300])
    N, S = int(bounds[-1]), 2400
    prop = rng.uniform(0.0, 1.0, (N, 22)).astype(np.float32)
    post = rng.integers(0, N, S)
    pre = rng.integers(0, N, S)
    kind = (rng.integers(0, 2, S) * 2).astype(np.uint8)
    w = rng.uniform(0.0, 1.0, (S, 2)).astype(np.float32)
    order = rng.permutation(S)
    d = str(tmp_path / "blocks")
    write_blocks(d, prop, bounds, post, pre, kind, w, order=order)

    for i in range(len(bounds) - 1):
        f = np.load(os.path.join(d, f"block_{i}.npz"))
        assert set(f.files) == set(KEYS)
        for k, dt in KEYS.items():
            assert f[k].dtype == dt, k
        assert f["property"].shape == (bounds[i + 1] - bounds[i], 22)
        assert f["weight"].shape == (len(f["output_neuron_idx"]), 2)

    p2, post2, pre2, kind2, w2 = load_npz_blocks(d)
    assert np.array_equal(p2, prop)
    assert len(post2) == S
    post_o, pre_o, kind_o, w_o = post[order], pre[order], kind[order], w[order]
    for n in range(N):
        a = np.nonzero(post_o == n)[0]
        b = np.nonzero(post2 == n)[0]
        assert np.array_equal(pre2[b], pre_o[a]), n
        assert np.array_equal(kind2[b], kind_o[a]), n
        assert np.array_equal(w2[b], w_o[a]), n
