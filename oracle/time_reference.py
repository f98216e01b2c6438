"""Test infrastructure: times the reference's own models/block.py (torch CPU) on the
single-block configuration (N=2000, K=100, dt=0.1 ms, p=0.01) in this container, for
the CPU-baseline statement beside the oracle port that bench.py times on the GPU box
(the reference tree is not there).  Usage: python oracle/time_reference.py [steps] [N]
"""
import os
import sys
import time

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path = [p for p in sys.path if os.path.abspath(p or ".") != HERE]   # the package, not this folder
REF = os.environ.get("DTB_REFERENCE")   # the reference checkout (yeyeleijun/Digital_twin_brain)
if not REF or not os.path.isdir(REF):
    sys.exit("set DTB_REFERENCE to a checkout of the reference, e.g. DTB_REFERENCE=/path/to/Digital_twin_brain python oracle/time_reference.py")
sys.path.insert(0, ROOT)
sys.path.insert(0, REF)

from oracle import oracle as O  # noqa: E402
from digital_twin_brain_b200 import synthetic  # noqa: E402
from models.block import block as RefBlock  # noqa: E402  (reference)


def main():
    steps = int(sys.argv[1]) if len(sys.argv) > 1 else 1000
    n = int(sys.argv[2]) if len(sys.argv) > 2 else 2000
    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    spec = synthetic.single_block(n, 100, name=f"ref_timing_{n}")
    rowptr, pre, kind, w = O.gen_network(spec.as_dict())
    post = np.repeat(np.arange(spec.N), spec.K)
    idx = np.stack([kind.astype(np.int64), post, pre.astype(np.int64)])
    idx = np.stack([idx, idx], axis=-1)
    idx[0, :, 1] += 1
    W = torch.sparse_coo_tensor(torch.from_numpy(idx.reshape(3, -1)), torch.from_numpy(w.reshape(-1).copy()),
                                (4, spec.N, spec.N))
    b = RefBlock(torch.from_numpy(spec.property()), W, delta_t=spec.dt)
    outdeg = np.bincount(pre, minlength=spec.N)
    for _ in range(3):
        b.run(noise_rate=0.01)
    events = 0
    t0 = time.perf_counter()
    for _ in range(steps):
        b.run(noise_rate=0.01)
        # propagated neurons are not kept by the reference; count the spikes' out-degrees plus
        # the expected noise share (p * N * K)
        events += int(outdeg[b.active.numpy()].sum()) + 0.01 * spec.N * spec.K
    dt = time.perf_counter() - t0
    print(f"reference models/block.py, torch {torch.__version__} CPU, {threads} threads, N={spec.N}, "
          f"K={spec.K}: {steps / dt:.1f} steps/s, {dt / steps * 1e3:.2f} ms/step, {events / dt:.3e} events/s")


if __name__ == "__main__":
    main()
