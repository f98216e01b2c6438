"""Ordered push: DTB_MODE_PULL propagated by scattering firing rows into
per-neuron slots summed in pull-row order must equal the row gather bit for
bit (and hence models/block.py's torch.sparse.mm order)."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from digital_twin_brain_b200 import Network, synthetic
from digital_twin_brain_b200._lib import (FIELD_ACTIVE, FIELD_I_SYN, FIELD_J, FIELD_T_LAST, FIELD_V,
                                          TUNE_PULL_METHOD)
from tests._helpers import GOLDEN, decay_like_reference, unpack
from tests.test_gpu_parity import class_decay_like_reference

pytestmark = pytest.mark.gpu

ROWS, SLOTS, MASKS, STREAM = 1, 2, 3, 4


def _state(net):
    return [net.get(f) for f in (FIELD_V, FIELD_J, FIELD_T_LAST, FIELD_I_SYN, FIELD_ACTIVE)]


@pytest.mark.parametrize("method", [SLOTS, MASKS, STREAM], ids=["slots", "masks", "stream"])
def test_ordered_push_matches_reference_golden(method):
    g = np.load(os.path.join(GOLDEN, "single_block_2k.npz"))
    spec = synthetic.config_single_block()
    net = Network.from_spec(spec, device=0, build_push=True, class_decay=class_decay_like_reference(spec))
    net.set_tuning(TUNE_PULL_METHOD, method)
    every = int(g["v_every"])
    act_ref = unpack(g["active"], spec.N)
    for c in range(int(g["steps"]) // every):
        s, m, na = net.run(every, noise_rate=0.01, mode="pull")
        assert np.array_equal(s, g["sums"][c * every:(c + 1) * every])
        assert np.array_equal(net.get(FIELD_V), g["V"][c])
        assert np.array_equal(net.get(FIELD_ACTIVE).astype(bool), act_ref[(c + 1) * every - 1])
    assert np.array_equal(net.get(FIELD_J), g["J_final"])
    assert np.array_equal(net.get(FIELD_I_SYN), g["I_syn_final"])


@pytest.mark.parametrize("method", [SLOTS, MASKS, STREAM], ids=["slots", "masks", "stream"])
@pytest.mark.parametrize("rate,K", [(0.01, 100), (0.05, 120), (0.3, 60)],
                         ids=["sparse", "overflowing_rows", "dense"])
def test_ordered_push_equals_row_gather(rate, K, method):
    """Slots: rows with more than 8 contributions per step fall back to the warp gather inside the same
    kernel.  Masks: one bit per pull-row position (in-degree up to 128)."""
    spec = synthetic.whole_brain(R=6, mean_size=700, sigma=0.5, K=K, gen_seed=3, name=f"wb6_K{K}")
    a = Network.from_spec(spec, device=0)
    b = Network.from_spec(spec, device=0)
    a.set_tuning(TUNE_PULL_METHOD, ROWS)
    b.set_tuning(TUNE_PULL_METHOD, method)
    for n in (1, 37, 64, 5):
        sa, ma, na = a.run(n, noise_rate=rate, mode="pull")
        sb, mb, nb = b.run(n, noise_rate=rate, mode="pull")
        assert np.array_equal(sa, sb) and np.array_equal(na, nb)
        np.testing.assert_array_equal(ma, mb)
        for x, y in zip(_state(a), _state(b)):
            assert np.array_equal(x, y)
    assert na.sum() > 0


def test_ordered_push_npz_positions_and_method_switches():
    """Host-built CSRs (file order inside rows) carry the pull-row positions into the push CSR;
    switching methods between runs keeps the state exact."""
    d = os.path.join(GOLDEN, "small_blocks")
    a = Network.from_npz(d, dt=0.1, seed=11, device=0)
    b = Network.from_npz(d, dt=0.1, seed=11, device=0)
    a.set_tuning(TUNE_PULL_METHOD, ROWS)
    for k, n in enumerate((20, 33, 7, 40, 11, 9, 13, 5)):
        b.set_tuning(TUNE_PULL_METHOD, (SLOTS, ROWS, MASKS, STREAM)[k % 4])
        sa, _, _ = a.run(n, noise_rate=0.02, mode="pull")
        sb, _, _ = b.run(n, noise_rate=0.02, mode="pull")
        assert np.array_equal(sa, sb)
        for x, y in zip(_state(a), _state(b)):
            assert np.array_equal(x, y)


def test_npz_hub_row_and_repeated_pairs(tmp_path):
    """A presynaptic hub longer than the device row sort (sorted on the host), pairs of neurons
    joined twice, rows in random file order: push rows ordered by (post, kind, pull-row position)
    and the ordered push still equals the row gather."""
    from digital_twin_brain_b200.generation import write_blocks
    rng = np.random.default_rng(5)
    N, K = 3000, 40
    rows = []
    for i in range(N):
        src = rng.choice(np.arange(1, N), K - 2, replace=False)
        src = np.concatenate([[0], src, [src[0]]])      # hub 0 in every row, one pair twice
        rng.shuffle(src)
        rows.append(src)
    post = np.repeat(np.arange(N), K)
    pre = np.concatenate(rows).astype(np.int64)
    pos = np.tile(np.arange(K), N)
    kind = np.where(pre >= 2400, 2, 0).astype(np.uint8)
    w = rng.random((N * K, 2)).astype(np.float32)
    spec = synthetic.config_single_block()
    prop = np.repeat(spec.class_property[:1], N, axis=0).copy()
    prop[2400:] = spec.class_property[1]
    prop[:, 3] = (np.arange(N) >= 1500).astype(np.float32)
    prop[:, 10:14] *= np.float32(2.5)
    write_blocks(str(tmp_path), prop.astype(np.float32), [0, 1500, N], post, pre, kind, w)
    a = Network.from_npz(str(tmp_path), dt=0.1, seed=2, device=0)
    qrp, qix, qw = a.get_csr("push")
    order = np.lexsort((pos, kind, post, pre))
    exp_rp = np.concatenate([[0], np.cumsum(np.bincount(pre, minlength=N))])
    assert np.array_equal(qrp, exp_rp) and qrp[1] - qrp[0] == N       # the hub's row is N long
    assert np.array_equal(qix, post[order].astype(np.uint32) | np.where(kind[order] == 2, np.uint32(0x80000000), 0))
    assert np.array_equal(qw, w[order])
    b = Network.from_npz(str(tmp_path), dt=0.1, seed=2, device=0)
    c = Network.from_npz(str(tmp_path), dt=0.1, seed=2, device=0)
    d = Network.from_npz(str(tmp_path), dt=0.1, seed=2, device=0)
    a.set_tuning(TUNE_PULL_METHOD, ROWS)
    b.set_tuning(TUNE_PULL_METHOD, SLOTS)
    c.set_tuning(TUNE_PULL_METHOD, MASKS)
    d.set_tuning(TUNE_PULL_METHOD, STREAM)
    for n in (50, 50):
        sa, _, na = a.run(n, noise_rate=0.05, mode="pull")
        for other in (b, c, d):
            so, _, no = other.run(n, noise_rate=0.05, mode="pull")
            assert np.array_equal(sa, so) and np.array_equal(na, no)
            for x, y in zip(_state(a), _state(other)):
                assert np.array_equal(x, y)


def test_masks_refused_beyond_128_inputs():
    from digital_twin_brain_b200._lib import DtbError
    spec = synthetic.single_block(600, 200, name="k200")
    net = Network.from_spec(spec, device=0)
    with pytest.raises(DtbError):
        net.set_tuning(TUNE_PULL_METHOD, MASKS)
    net.run(20, noise_rate=0.02, mode="pull")      # auto: slots (in-degree 200 > 128)
