"""Failure paths of the C ABI (no GPU needed: every case here is refused before the
library touches a device).  The reference aborts the process on such input
(cuda/src/common.cpp:187-230 prints and calls exit); the library returns a status
code and keeps the reason for dtb_last_error instead, and the process goes on.
"""
import os
import shutil
import zipfile

import numpy as np
import pytest

from digital_twin_brain_b200 import Network, synthetic
from digital_twin_brain_b200._lib import DtbError
from tests._helpers import GOLDEN

ARG, FORMAT, IO = 1, 5, 4


def _blocks(tmp_path):
    d = str(tmp_path / "blocks")
    shutil.copytree(os.path.join(GOLDEN, "small_blocks"), d)
    return d


def test_missing_directory():
    with pytest.raises(DtbError) as e:
        Network.from_npz("/nonexistent/dtb-blocks", dt=0.1)
    assert e.value.code == IO and "no block_0.npz" in str(e.value)


def test_truncated_npz(tmp_path):
    d = _blocks(tmp_path)
    path = os.path.join(d, "block_1.npz")
    size = os.path.getsize(path)
    with open(path, "r+b") as f:
        f.truncate(size // 2)
    with pytest.raises(DtbError) as e:
        Network.from_npz(d, dt=0.1)
    assert e.value.code == FORMAT and "end-of-central-directory" in str(e.value)


@pytest.mark.parametrize("member", ["property.npy", "output_neuron_idx.npy"])
def test_corrupt_zip_member(tmp_path, member):
    """One byte flipped inside a member's data: caught by its CRC-32."""
    d = _blocks(tmp_path)
    path = os.path.join(d, "block_0.npz")
    with zipfile.ZipFile(path) as z:
        info = z.getinfo(member)
    with open(path, "r+b") as f:
        f.seek(info.header_offset + 26)
        name_len = int.from_bytes(f.read(2), "little")
        extra_len = int.from_bytes(f.read(2), "little")
        at = info.header_offset + 30 + name_len + extra_len + info.compress_size - 5
        f.seek(at)
        b = f.read(1)
        f.seek(at)
        f.write(bytes([b[0] ^ 0x5A]))
    with pytest.raises(DtbError) as e:
        Network.from_npz(d, dt=0.1)
    assert e.value.code == FORMAT
    assert "CRC-32 mismatch" in str(e.value) or "deflate" in str(e.value)


def test_npz_with_wrong_property_shape(tmp_path):
    d = _blocks(tmp_path)
    path = os.path.join(d, "block_2.npz")
    with np.load(path) as z:
        arrays = {k: z[k] for k in z.files}
    arrays["property"] = arrays["property"][:, :21]
    np.savez(path, **arrays)
    with pytest.raises(DtbError) as e:
        Network.from_npz(d, dt=0.1)
    assert e.value.code == FORMAT and "float32 [N,22]" in str(e.value)


def _arrays(N=50, K=4, seed=0):
    rng = np.random.default_rng(seed)
    spec = synthetic.single_block(N, K)
    prop = spec.property()
    post = np.repeat(np.arange(N), K).astype(np.uint32)
    pre = rng.integers(0, N, N * K).astype(np.uint32)
    kind = np.where(pre >= int(0.8 * N), 2, 0).astype(np.uint8)
    w = rng.random((N * K, 2)).astype(np.float32)
    return prop, post, pre, kind, w


def test_presynaptic_index_out_of_range():
    prop, post, pre, kind, w = _arrays()
    pre[17] = 50                                # N = 50
    with pytest.raises(DtbError) as e:
        Network.from_arrays(prop, post, pre, kind, w, dt=0.1)
    assert e.value.code == ARG and "synapse 17 references neuron out of range" in str(e.value)


def test_bad_receptor_kind():
    prop, post, pre, kind, w = _arrays()
    kind[3] = 1
    with pytest.raises(DtbError) as e:
        Network.from_arrays(prop, post, pre, kind, w, dt=0.1)
    assert e.value.code == ARG and "kind must be 0 or 2" in str(e.value)


@pytest.mark.parametrize("col", [4, 8, 18])
def test_nan_property(col):
    prop, post, pre, kind, w = _arrays()
    prop[7, col] = np.nan
    with pytest.raises(DtbError) as e:
        Network.from_arrays(prop, post, pre, kind, w, dt=0.1)
    assert e.value.code == ARG and f"property row 7 column {col} is NaN" in str(e.value)


def test_infinite_threshold_allowed_in_checks():
    """+inf (a neuron that never fires, as the ensemble pad neurons) is not refused by the NaN
    check; such a network then only fails later for the lack of a GPU, not for its values."""
    prop, post, pre, kind, w = _arrays()
    prop[7, 8] = np.inf
    try:
        Network.from_arrays(prop, post, pre, kind, w, dt=0.1)
    except DtbError as e:
        assert "NaN" not in str(e)


def test_nonpositive_dt_and_sizes():
    prop, post, pre, kind, w = _arrays()
    with pytest.raises(DtbError):
        Network.from_arrays(prop[:0], post[:0], pre[:0], kind[:0], w[:0], dt=0.1)
