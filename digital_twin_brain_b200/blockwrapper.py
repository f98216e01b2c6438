"""In-process GPU backend with the interface of the reference's gRPC client
``BlockWrapper`` (cuda/python/dist_blockwrapper_pytorch.py:30-541), so that
the reference's drivers (simulation/simulation.py, data_assimilation/
DataAssimilation.py) can drive the B200 block directly:

    from digital_twin_brain_b200.blockwrapper import BlockWrapper
    block_model = BlockWrapper(address, path, delta_t)          # address: unused

Same method names, argument meaning and return types: ``run`` is a generator
of per-step tuples of CUDA tensors (freqs int32 [n_subblk], vmean, sample
spikes uint8 and V, imean), ``mul_property_by_subblk`` sets a column of a
subblock to (base x value) unless ``accumulate``, ``gamma_property_by_subblk``
draws per-neuron Gamma(alpha, beta) values, ``set_samples`` selects the neurons
``run`` reports, ``update_property`` writes single (neuron, column) entries.

Differences, by design:
  * ``path`` is a directory of block_{i}.npz files (generation/make_block.py
    format, read as generation/read_block.py:12-97 reads them); there is no
    server, route table or rebasing of subblock ids across blocks: column 3 of
    the property matrix is the global subblock id.
  * The block follows models/block.py (initial V = (V_th + V_reset) / 2, every
    neuron counted in the subblock statistics); the noise rate is the
    per-neuron column 0 of the property matrix, as on the reference's server
    (cuda/src/stage/spike.cpp:157).
  * ``update_property`` rebuilds the parameters from the files' property matrix
    plus every entry written through it so far: gamma draws and subblock
    scalings applied before it are replaced (the client resets its scaling
    record at the same point, dist_blockwrapper_pytorch.py:355).
  * ``imean`` steps one step at a time (the mean synaptic current of every
    subblock is taken from the device state after each step).
"""
from __future__ import annotations

import os
import time
import zipfile
from collections import OrderedDict

import numpy as np
import torch

from .network import Network
from ._lib import FIELD_I_SYN, FIELD_SUB_COUNT, DTB_DEVICE, DTB_HOST
from . import _lib


def _npz_rows(path: str) -> int:
    """Rows of the `property` array of an npz file, read from the .npy header only."""
    with zipfile.ZipFile(path) as z, z.open("property.npy") as f:
        version = np.lib.format.read_magic(f)
        read = np.lib.format.read_array_header_1_0 if version == (1, 0) else np.lib.format.read_array_header_2_0
        shape, _, _ = read(f)
    return int(shape[0])


class BlockWrapper:
    """cuda/python/dist_blockwrapper_pytorch.py:30 BlockWrapper, served by libdtb in this process."""

    # 22-column property index -> the server's property id (-1: not a parameter)
    property_idx_trans = torch.tensor([19, -1, 0, -1, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18],
                                      dtype=torch.int64)
    buffersize = 1024 ** 3 // 4

    def __init__(self, address, path, delta_t, route_path=None, print_stat=False, force_rebase=False,
                 allow_rebase=True, overlap=2, *, device: int = 0, seed: int = 0, build_push: bool = True,
                 mode: str = "auto"):
        self.print_stat = print_stat
        self._mode = mode
        self._path = path
        self._dev = torch.device("cuda", device)
        files = []
        while os.path.exists(os.path.join(path, f"block_{len(files)}.npz")):
            files.append(os.path.join(path, f"block_{len(files)}.npz"))
        assert files, f"no block_0.npz in {path}"
        self._files = files
        self._net = Network.from_npz(path, dt=float(delta_t), seed=seed, device=device, build_push=build_push)
        n_sub = self._net.n_sub
        counts = np.empty(max(n_sub, 1), np.uint32)
        if n_sub:
            _lib.call("dtb_block_get", self._net._h, FIELD_SUB_COUNT, counts.ctypes.data_as(_lib.c_vp), DTB_HOST)
        present = np.nonzero(counts[:n_sub] > 0)[0]
        self._block_id = torch.arange(len(files), dtype=torch.int64, device=self._dev)
        self._neurons_per_block = torch.tensor([_npz_rows(f) for f in files], dtype=torch.int64, device=self._dev)
        self._neurons_thrush = torch.cat([torch.zeros(1, dtype=torch.int64, device=self._dev),
                                          torch.cumsum(self._neurons_per_block, 0)])
        self._subblk_id = torch.from_numpy(present.astype(np.int64)).to(self._dev)
        self._neurons_per_subblk = torch.from_numpy(counts[present].astype(np.int64)).to(self._dev)
        self._buff_len = max(1, min(4096, self.buffersize // max(1, len(present))))
        self._last_hp = {}               # (subblk id, column) -> value last set (1 = base)
        self._prop = None                # host property matrix, loaded by update_property / imean
        self._sub_of = None
        self._sample_num = 0
        self._iterations = 0
        self._last_run_s = 0.0

    # ------------------------------------------------------------ properties
    @property
    def total_neurons(self):
        return self._neurons_per_block.sum()

    @property
    def block_id(self):
        return self._block_id

    @property
    def subblk_id(self):
        return self._subblk_id

    @property
    def total_subblks(self):
        return self._subblk_id.shape[0]

    @property
    def neurons_per_subblk(self):
        return self._neurons_per_subblk

    @property
    def neurons_per_block(self):
        return self._neurons_per_block

    @property
    def network(self) -> Network:
        """The underlying libdtb network handle."""
        return self._net

    # ------------------------------------------------------------ stepping
    def _property(self) -> np.ndarray:
        if self._prop is None:
            self._prop = np.concatenate([np.load(f)["property"] for f in self._files]).astype(np.float32)
        return self._prop

    def _imean(self) -> torch.Tensor:
        if self._sub_of is None:
            sub = self._property()[:, 3].astype(np.int64)
            self._sub_of = torch.from_numpy(sub).to(self._dev)
            self._sub_valid = (self._sub_of >= 0) & (self._sub_of < self._net.n_sub)
        isyn = torch.empty(self._net.N, dtype=torch.float32, device=self._dev)
        self._net._torch_ready()
        _lib.call("dtb_block_get", self._net._h, FIELD_I_SYN, _lib.c_vp(isyn.data_ptr()), DTB_DEVICE)
        self._net.synchronize()
        acc = torch.zeros(max(self._net.n_sub, 1), dtype=torch.float64, device=self._dev)
        acc.index_add_(0, self._sub_of[self._sub_valid], isyn[self._sub_valid].double())
        return (acc[self._subblk_id] / self._neurons_per_subblk.double()).float()

    def run(self, iterations, freqs=True, vmean=False, sample_for_show=False, imean=False, strategy=None):
        """dist_blockwrapper_pytorch.py:213-316: yields, per step, the tuple of the requested outputs
        (freqs int32 [n_subblk], vmean f32 [n_subblk], spikes uint8 [n_sample], V f32 [n_sample],
        imean f32 [n_subblk]) as CUDA tensors."""
        assert not sample_for_show or self._sample_num > 0, "set_samples first"
        t0 = time.perf_counter()
        done = 0
        while done < iterations:
            n = 1 if imean else min(self._buff_len, iterations - done)
            s, mn, _ = self._net.run(n, noise_rate=None, mode=self._mode, out="device")
            outs = []
            if freqs:
                outs.append(s.index_select(1, self._subblk_id).round().to(torch.int32))
            if vmean:
                outs.append(mn.index_select(1, self._subblk_id))
            if sample_for_show:
                sp, v = self._net.get_samples(out="device")
                outs.append(sp[-n:])
                outs.append(v[-n:])
            if imean:
                outs.append(self._imean().unsqueeze(0))
            done += n
            self._iterations += n
            for j in range(n):
                yield tuple(o[j] for o in outs)
        self._last_run_s = time.perf_counter() - t0

    # ------------------------------------------------------------ parameters
    @staticmethod
    def _check_idx(property_idx, values):
        assert isinstance(property_idx, torch.Tensor) and isinstance(values, torch.Tensor)
        assert property_idx.dtype == torch.int64 and values.dtype == torch.float32
        assert len(property_idx.shape) == 2 and property_idx.shape[1] == 2
        assert values.shape[0] == property_idx.shape[0]
        trans = BlockWrapper.property_idx_trans[property_idx[:, 1].cpu()]
        assert (trans >= 0).all(), "columns 1 and 3 are not parameters"

    def update_property(self, property_idx, property_weight, bid=None):
        """dist_blockwrapper_pytorch.py:317-380: property[neuron, column] = weight for every row."""
        self._check_idx(property_idx, property_weight)
        idx = property_idx.cpu().numpy()
        w = property_weight.cpu().numpy()
        if bid is not None:
            assert 0 <= bid < len(self._files)
            idx = idx.copy()
            idx[:, 0] += int(self._neurons_thrush[bid])
        prop = self._property()
        assert (idx[:, 0] >= 0).all() and (idx[:, 0] < prop.shape[0]).all()
        prop[idx[:, 0], idx[:, 1]] = w          # later rows win, as the server applies them in order
        self._net.update_property(prop)
        self._last_hp.clear()

    def mul_property_by_subblk(self, property_idx, property_hyper_parameter, accumulate=False):
        """dist_blockwrapper_pytorch.py:446-458: column of subblock <- base x value (x the previous
        value as well when accumulate)."""
        self._check_idx(property_idx, property_hyper_parameter)
        idx = property_idx.cpu().numpy()
        hp = property_hyper_parameter.cpu().numpy().astype(np.float32)
        vals = np.empty(len(hp), np.float32)
        for i, (sb, col) in enumerate(idx):
            key = (int(sb), int(col))
            v = hp[i] * self._last_hp.get(key, np.float32(1.0)) if accumulate else hp[i]
            self._last_hp[key] = np.float32(v)
            vals[i] = v
        self._net.scale_property_by_subblock(idx[:, 0], idx[:, 1], vals)
        if self.print_stat:
            print("property_hyper_parameter", float(hp.max()), float(hp.min()), float(hp.mean()))

    def gamma_property_by_subblk(self, property_idx, gamma_concentration, gamma_rate, debug=False):
        """dist_blockwrapper_pytorch.py:460-501: every neuron of the subblock draws its own
        Gamma(concentration, rate) value of the column."""
        assert len(gamma_rate.shape) == 1
        if gamma_concentration is None:
            gamma_concentration = torch.ones_like(gamma_rate)
        assert len(gamma_concentration.shape) == 1
        self._check_idx(property_idx, gamma_rate.float())
        assert (gamma_concentration >= 0).all() and (gamma_rate >= 0).all()
        idx = property_idx.cpu().numpy()
        a = gamma_concentration.cpu().numpy().astype(np.float32)
        b = gamma_rate.cpu().numpy().astype(np.float32)
        self._net.gamma_property_by_subblock(idx[:, 0], idx[:, 1], a, b)
        for sb, col in idx:
            self._last_hp[(int(sb), int(col))] = np.float32(1.0)
        if debug:
            g = self._net.g_factors()
            sub = self._property()[:, 3].astype(np.int64)
            for (sb, col), al, be in zip(idx, a, b):
                if not 10 <= col < 14:
                    continue
                val = g[sub == sb, col - 10]
                mean_error = abs(val.mean() - al / be) / (al / be)
                var_error = abs(val.var() - al / be ** 2) / (al / be ** 2)
                print("brain_id: {}, prop_id: {}, mean_err: {:.2f}, var_err: {:.2f}".format(
                    sb, self.property_idx_trans[col].item(), mean_error, var_error))
        return True

    def set_samples(self, sample_idx, bid=None):
        """dist_blockwrapper_pytorch.py:503-525: the neurons whose spike and V ``run`` reports, in the given order."""
        assert isinstance(sample_idx, torch.Tensor) and len(sample_idx.shape) == 1
        assert sample_idx.dtype == torch.int64
        idx = sample_idx.cpu().numpy()
        if bid is not None:
            idx = idx + int(self._neurons_thrush[bid])
        self._net.set_samples(idx.astype(np.uint32), self._buff_len)
        self._sample_num = len(idx)

    # ------------------------------------------------------------ bookkeeping
    def last_time_stat(self):
        """dist_blockwrapper_pytorch.py:146-186, reduced to what one process measures: the wall time of
        the last ``run`` (no routing or reporting stages)."""
        import pandas as pd
        rows = ["computing_duration", "routing_duration", "reporting_duration", "duration_inter_node",
                "duration_intra_node", "sending_byte_size_inter_node", "sending_byte_size_intra_node",
                "recving_byte_size_inter_node", "recving_byte_size_intra_node"]
        data = np.zeros((1, 1, len(rows)))
        data[0, 0, 0] = self._last_run_s
        col = OrderedDict([("total_mean", np.mean), ("total_std", np.std)])
        table = pd.DataFrame(np.array([[f(data[:, :, i]) for f in col.values()] for i in range(len(rows))]),
                             index=pd.Index(rows), columns=list(col.keys()))
        return data, table

    def close(self):
        if self._net is not None:
            self._net.close()
            self._net = None

    def shutdown(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, exc_type, exc_val, exc_tb):
        self.close()
