"""Block files in the reference's on-disk layout.

``write_blocks`` writes a network as ``block_{i}.npz`` files, one per
population, with the keys and dtypes of ``generation/make_block.py:473-479``
(``property`` f32[n,22], ``output_neuron_idx`` u32, ``input_block_idx`` i16
relative to the file's own index, ``input_neuron_idx`` u32 local to the source
population, ``input_channel_offset`` u8, ``weight`` f32[E,2]).  The reference's
``generation/read_block.py:connect_for_block`` reads them back, and so does
``Network.from_npz`` (the C++ reader in libdtb).
"""
from __future__ import annotations

import os

import numpy as np


def write_blocks(directory: str, property: np.ndarray, bounds, post, pre, kind, weight, order=None):
    """Write populations [bounds[i], bounds[i+1]) as block_i.npz.

    Synapses are written grouped by postsynaptic population, keeping their
    given order (``order`` optionally permutes them first), so that the file
    order inside every postsynaptic row is the order given here.
    """
    os.makedirs(directory, exist_ok=True)
    bounds = np.asarray(bounds, np.int64)
    post = np.asarray(post, np.int64)
    pre = np.asarray(pre, np.int64)
    kind = np.asarray(kind, np.uint8)
    weight = np.asarray(weight, np.float32).reshape(-1, 2)
    if order is not None:
        post, pre, kind, weight = post[order], pre[order], kind[order], weight[order]
    pop_post = np.searchsorted(bounds, post, side="right") - 1
    pop_pre = np.searchsorted(bounds, pre, side="right") - 1
    for i in range(len(bounds) - 1):
        sel = np.nonzero(pop_post == i)[0]
        sel = sel[np.argsort(post[sel], kind="stable")]
        np.savez(os.path.join(directory, f"block_{i}"),
                 property=np.ascontiguousarray(property[bounds[i]:bounds[i + 1]], np.float32),
                 output_neuron_idx=np.ascontiguousarray(post[sel] - bounds[i], np.uint32),
                 input_block_idx=np.ascontiguousarray(pop_pre[sel] - i, np.int16),
                 input_neuron_idx=np.ascontiguousarray(pre[sel] - bounds[pop_pre[sel]], np.uint32),
                 input_channel_offset=np.ascontiguousarray(kind[sel], np.uint8),
                 weight=np.ascontiguousarray(weight[sel], np.float32))


def write_population(directory: str, i: int, bounds, property_rows: np.ndarray, post_local, pre, kind, weight):
    """Write population i alone as block_i.npz (the layout of write_blocks), from its synapses:
    post_local (postsynaptic index inside the population, in the order to keep), pre (global
    presynaptic index), kind, weight [E,2].  Writing a large network population by population
    keeps host memory at one population's synapses."""
    os.makedirs(directory, exist_ok=True)
    bounds = np.asarray(bounds, np.int64)
    pre = np.asarray(pre, np.int64)
    pop_pre = np.searchsorted(bounds, pre, side="right") - 1
    np.savez(os.path.join(directory, f"block_{i}"),
             property=np.ascontiguousarray(property_rows, np.float32),
             output_neuron_idx=np.ascontiguousarray(post_local, np.uint32),
             input_block_idx=np.ascontiguousarray(pop_pre - i, np.int16),
             input_neuron_idx=np.ascontiguousarray(pre - bounds[pop_pre], np.uint32),
             input_channel_offset=np.ascontiguousarray(kind, np.uint8),
             weight=np.ascontiguousarray(np.asarray(weight, np.float32).reshape(-1, 2)))
