"""The BlockWrapper adapter (cuda/python/dist_blockwrapper_pytorch.py:30-541)
driving libdtb, against the oracle: per-step subblock spike counts and mean V,
sampled spikes and V, subblock scaling and gamma draws."""
import ctypes
import ctypes.util
import os

import numpy as np
import pytest
import torch

from oracle import oracle as O
from digital_twin_brain_b200.blockwrapper import BlockWrapper
from tests._helpers import GOLDEN, load_npz_blocks

pytestmark = pytest.mark.gpu

DIR = os.path.join(GOLDEN, "small_blocks")
_libm = ctypes.CDLL(ctypes.util.find_library("m"))
_libm.expf.restype = ctypes.c_float
_libm.expf.argtypes = [ctypes.c_float]


def native_decay(prop, dt):
    """exp(-dt/tau) as the library derives it from a file's property matrix (expf of fl(1/tau) * -dt)."""
    r = (np.float32(1) / prop[:, 18:22].astype(np.float32)) * np.float32(-dt)
    return np.vectorize(lambda x: _libm.expf(float(x)), otypes=[np.float32])(r).T.copy()


def _oracle(seed, dt):
    prop, post, pre, kind, w = load_npz_blocks(DIR)
    rp, opre, okind, ow = O.pull_csr(prop.shape[0], post, pre, kind, w)
    return prop, O.OracleBlock(prop, native_decay(prop, dt), rp, opre, okind, ow, dt, seed)


def test_blockwrapper_run_matches_oracle():
    dt, seed = 0.1, 11
    prop, ob = _oracle(seed, dt)
    bw = BlockWrapper("unused:0", DIR, dt, seed=seed, mode="pull")
    N = prop.shape[0]
    assert int(bw.total_neurons) == N
    sub = prop[:, 3].astype(int)
    ids = np.unique(sub)
    assert np.array_equal(bw.subblk_id.cpu().numpy(), ids)
    assert np.array_equal(bw.neurons_per_subblk.cpu().numpy(), np.bincount(sub)[ids])
    sample = torch.tensor([N - 1, 0, 7, 123, 7], dtype=torch.int64)
    bw.set_samples(sample)
    steps = 0
    for chunk in (50, 130):
        for out in bw.run(chunk, freqs=True, vmean=True, sample_for_show=True):
            f, vm, sp, v = out
            assert f.dtype == torch.int32 and f.is_cuda and sp.dtype == torch.uint8
            so, mo = ob.run(None)                        # per-neuron noise rate (property column 0)
            assert np.array_equal(f.cpu().numpy(), so[ids].astype(np.int32)), f"step {steps}"
            np.testing.assert_allclose(vm.cpu().numpy(), mo[ids], rtol=2e-6)
            assert np.array_equal(sp.cpu().numpy(), ob.active[sample.numpy()])
            assert np.array_equal(v.cpu().numpy(), ob.V[sample.numpy()])
            steps += 1
    assert steps == 180


def test_blockwrapper_imean_and_properties():
    dt, seed = 0.1, 3
    prop, ob = _oracle(seed, dt)
    bw = BlockWrapper("unused:0", DIR, dt, seed=seed, mode="pull")
    sub = prop[:, 3].astype(int)
    ids = np.unique(sub)
    for (f, im) in bw.run(20, freqs=True, imean=True):
        ob.run(None)
        want = np.array([ob.Isyn[sub == i].astype(np.float64).mean() for i in ids])
        np.testing.assert_allclose(im.cpu().numpy(), want, rtol=1e-5, atol=1e-6)
    # mul_property_by_subblk: not accumulated -> base x value; accumulated -> previous x value
    idx = torch.tensor([[int(ids[0]), 10]], dtype=torch.int64)
    bw.mul_property_by_subblk(idx, torch.tensor([2.0]))
    bw.mul_property_by_subblk(idx, torch.tensor([1.5]))                    # 1.5 x base, not 3 x base
    bw.mul_property_by_subblk(idx, torch.tensor([2.0]), accumulate=True)   # 3 x base
    p2 = prop.copy()
    p2[sub == ids[0], 10] = prop[sub == ids[0], 10] * np.float32(3.0)
    ob.P = O.Params.from_property(p2, native_decay(p2, dt))
    for (f,) in bw.run(40):
        so, _ = ob.run(None)
        assert np.array_equal(f.cpu().numpy(), so[ids].astype(np.int32))
    assert np.array_equal(bw.network.get(0), ob.V)
    # update_property of single entries (neuron, column)
    pidx = torch.tensor([[5, 8], [6, 2]], dtype=torch.int64)
    bw.update_property(pidx, torch.tensor([-52.0, 0.5]))
    with pytest.raises(AssertionError):
        bw.update_property(torch.tensor([[5, 3]], dtype=torch.int64), torch.tensor([1.0]))
    # gamma draws: one value per neuron, mean / variance of Gamma(5, 5)
    big = torch.tensor([[int(i), 11] for i in ids], dtype=torch.int64)
    assert bw.gamma_property_by_subblk(big, torch.full((len(ids),), 5.0), torch.full((len(ids),), 5.0))
    g = bw.network.g_factors()[:, 1]
    assert abs(g.mean() - 1.0) < 0.1 and abs(g.var() - 0.2) < 0.1
    bw.close()
