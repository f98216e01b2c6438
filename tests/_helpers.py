"""Shared helpers of the test-suite (not a test module)."""
import os

import numpy as np
import torch

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def unpack(bits: np.ndarray, n: int) -> np.ndarray:
    return np.unpackbits(bits, axis=-1, bitorder="little")[..., :n].astype(bool)


def decay_like_reference(prop: np.ndarray, dt: float) -> np.ndarray:
    """exp(-dt/tau) exactly as models/block.py:71 evaluates it, as [4, N]."""
    tau = torch.from_numpy(np.ascontiguousarray(prop, np.float32)).transpose(0, 1)[18:22]
    return torch.exp(-dt / tau).numpy().copy()


def load_npz_blocks(directory: str):
    """Global COO (post, pre, kind, w) in file order + property, as read_block.py concatenates them."""
    files = []
    i = 0
    while os.path.exists(os.path.join(directory, f"block_{i}.npz")):
        files.append(np.load(os.path.join(directory, f"block_{i}.npz")))
        i += 1
    bases = np.concatenate([[0], np.cumsum([f["property"].shape[0] for f in files])]).astype(np.int64)
    props, posts, pres, kinds, ws = [], [], [], [], []
    for i, f in enumerate(files):
        props.append(f["property"])
        po, pr, k, w = O.coo_from_npz_arrays(f["output_neuron_idx"], f["input_block_idx"], f["input_neuron_idx"],
                                             f["input_channel_offset"], f["weight"], i, bases)
        posts.append(po); pres.append(pr); kinds.append(k); ws.append(w)
    return (np.concatenate(props), np.concatenate(posts), np.concatenate(pres), np.concatenate(kinds),
            np.concatenate(ws))


def schedule_steps(schedule):
    for n, rate, iso in schedule:
        for _ in range(int(n)):
            yield float(rate), bool(iso)
