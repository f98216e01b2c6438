"""The npz loader (generation/read_block.py:12-97 layout, cuda/src/configuration.cpp:214-341,
575-828 roles) on the whole-brain network structure written as one block file per region:
pull rows bit-exact against the generator's rows (sampled everywhere), the device-built push
CSR's row lengths against the out-degrees counted over every pull entry, and the load time.
The size is the whole-brain structure scaled by DTB_NPZ_SCALE (default 0.05; 1.0 writes about
45 GB of files)."""
import os
import time

import numpy as np
import pytest
import torch

from oracle import oracle as O
from digital_twin_brain_b200 import Network, synthetic
from digital_twin_brain_b200.generation import write_population

pytestmark = [pytest.mark.gpu, pytest.mark.slow]
KIND = np.uint32(0x80000000)


def write_whole_brain_blocks(directory, spec):
    d = spec.as_dict()
    rs = np.asarray(spec.region_start, np.int64)
    prop = spec.class_property
    cls = spec.neuron_class()
    for r in range(spec.R):
        n0, n1 = int(rs[r]), int(rs[r + 1])
        pre, kind, w = O.gen_rows(d, n0, n1)
        post_local = np.repeat(np.arange(n1 - n0, dtype=np.uint32), spec.K)
        write_population(directory, r, rs, prop[cls[n0:n1]], post_local, pre, kind, w)


def test_whole_brain_npz_load(tmp_path):
    scale = float(os.environ.get("DTB_NPZ_SCALE", "0.05"))
    spec = synthetic.config_whole_brain(scale=scale)
    d = str(tmp_path / "blocks")
    t0 = time.perf_counter()
    write_whole_brain_blocks(d, spec)
    t_write = time.perf_counter() - t0
    nbytes = sum(os.path.getsize(os.path.join(d, f)) for f in os.listdir(d))
    t0 = time.perf_counter()
    net = Network.from_npz(d, dt=0.1, seed=0, device=0, build_push=True)
    net.synchronize()
    t_load = time.perf_counter() - t0
    print(f"\nnpz whole-brain x{scale}: N={spec.N} S={spec.S} files={spec.R} bytes={nbytes} "
          f"write_s={t_write:.1f} load_s={t_load:.2f} ({nbytes / t_load / 1e9:.2f} GB/s of files)")
    assert net.N == spec.N and net.S == spec.S
    K = spec.K
    rp = net.get_csr_rowptr("pull")
    assert np.array_equal(rp, np.arange(spec.N + 1, dtype=np.int64) * K)
    rng = np.random.default_rng(0)
    rows = np.unique(np.concatenate([rng.integers(0, spec.N, 300), spec.region_start[:-1],
                                     spec.region_start[1:] - 1, [spec.N - 1]]))
    dd = spec.as_dict()
    for r in rows:
        ix, w = net.get_csr_entries("pull", int(r) * K, K)
        pre, kind, ow = O.gen_rows(dd, int(r), int(r) + 1)
        assert np.array_equal(ix, pre | np.where(kind == 2, KIND, np.uint32(0))), f"row {r}"
        assert np.array_equal(w, ow)
    qrp = net.get_csr_rowptr("push")
    counts = torch.zeros(spec.N, dtype=torch.int64, device="cuda:0")
    chunk = 1 << 27
    for e0 in range(0, net.S, chunk):
        ix, _ = net.get_csr_entries("pull", e0, min(chunk, net.S - e0), device=True, weights=False)
        counts += torch.bincount((ix & 0x7FFFFFFF).to(torch.int64), minlength=spec.N)
    assert np.array_equal(np.diff(qrp), counts.cpu().numpy())
    s, _, _ = net.run(80, noise_rate=0.01, mode="push")
    assert s[60:].sum() > 0


def test_npz_error_in_a_loader_thread(tmp_path):
    """A corrupt member that only the second pass reads (the weights of one of 12 files): the
    worker thread that meets it stops the load, and the caller gets DTB_ERR_FORMAT naming the
    member; the library stays usable and the rewritten files then load."""
    import zipfile
    from digital_twin_brain_b200._lib import DtbError
    spec = synthetic.whole_brain(R=12, mean_size=800, sigma=0.3, K=30, gen_seed=3, name="wb12")
    d = str(tmp_path / "blocks")
    write_whole_brain_blocks(d, spec)
    path = os.path.join(d, "block_7.npz")
    with zipfile.ZipFile(path) as z:
        info = z.getinfo("weight.npy")
    with open(path, "r+b") as f:
        f.seek(info.header_offset + 26)
        skip = int.from_bytes(f.read(2), "little") + int.from_bytes(f.read(2), "little")
        at = info.header_offset + 30 + skip + info.compress_size // 2
        f.seek(at)
        b = f.read(1)
        f.seek(at)
        f.write(bytes([b[0] ^ 0xFF]))
    with pytest.raises(DtbError) as e:
        Network.from_npz(d, dt=0.1, device=0)
    assert e.value.code == 5 and "weight" in str(e.value)
    write_whole_brain_blocks(d, spec)
    net = Network.from_npz(d, dt=0.1, device=0)
    assert net.N == spec.N and net.S == spec.S
