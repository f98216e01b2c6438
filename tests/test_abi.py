"""The C-ABI library builds, loads and exports every entry point include/dtb.h declares
(no GPU needed: nothing here launches a kernel)."""
import ctypes
import os
import re

import numpy as np
import pytest

from digital_twin_brain_b200 import _lib, build, synthetic
from digital_twin_brain_b200.models.block import coo_entries
from tests._helpers import ROOT


def declared_functions():
    src = open(os.path.join(ROOT, "include", "dtb.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*int\s+(dtb_\w+)\s*\(", src, flags=re.M)))


def test_header_declares_the_api():
    names = declared_functions()
    for required in ("dtb_block_create", "dtb_block_run", "dtb_block_get", "dtb_bold_run", "dtb_last_error",
                     "dtb_block_create_from_npz", "dtb_block_create_synthetic", "dtb_block_save"):
        assert required in names


def test_library_exports_every_declared_symbol():
    path = build.build()
    L = ctypes.CDLL(path)
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing
    assert set(declared_functions()) <= set(_lib._SIGS)


def test_library_is_sm100a_and_reports_errors_without_gpu():
    L = _lib.load()
    assert L.dtb_abi_version() == 1
    h = ctypes.c_void_p()
    rc = L.dtb_block_create(None, ctypes.byref(h))
    assert rc == 1 and "null" in _lib.last_error()
    # nvcc target recorded in the build flags
    assert "arch=compute_100a,code=sm_100a" in " ".join(build.NVCC_FLAGS)


def test_coo_pairs_from_read_block_layout():
    import torch
    post = np.array([0, 0, 1, 2])
    pre = np.array([3, 1, 2, 0])
    kind = np.array([0, 2, 0, 2], np.uint8)
    w = np.arange(8, dtype=np.float32).reshape(4, 2)
    idx = np.stack([kind.astype(np.int64), post, pre])
    idx = np.stack([idx, idx], -1)
    idx[0, :, 1] += 1
    W = torch.sparse_coo_tensor(torch.from_numpy(idx.reshape(3, -1)), torch.from_numpy(w.reshape(-1)), (4, 4, 4))
    p, q, k, ww = coo_entries(W)
    assert np.array_equal(p, post) and np.array_equal(q, pre) and np.array_equal(k, kind) and np.array_equal(ww, w)


def test_coo_generic_entries_keep_channel_order():
    import torch
    idx = torch.tensor([[1, 3, 0], [0, 0, 1], [2, 1, 0]])
    W = torch.sparse_coo_tensor(idx, torch.tensor([5.0, 6.0, 7.0]), (4, 3, 3))
    p, q, k, ww = coo_entries(W)
    assert list(p) == [0, 0, 1] and list(q) == [2, 1, 0] and list(k) == [0, 2, 0]
    assert ww.tolist() == [[0.0, 5.0], [0.0, 6.0], [7.0, 0.0]]


def test_synthetic_specs():
    s0 = synthetic.config_single_block()
    assert s0.N == 2000 and s0.K == 100 and s0.region_n_exc[0] == 1600
    p = s0.property()
    assert p.shape == (2000, 22) and set(np.unique(p[:, 3])) == {0.0, 1.0}
    assert np.allclose(p[0, 10:14], [0.01, 0.0005, 0.1, 0.005]) and p[0, 8] == -50 and p[0, 9] == -55
    s2 = synthetic.config_whole_brain()
    assert s2.R == 90 and 1.5e7 < s2.N < 3e7 and abs(s2.S - 100 * s2.N) == 0
    assert np.allclose(s2.cum[:, -1], 1.0) and (np.diff(s2.cum, axis=1) >= 0).all()


def declared_constants():
    """Every `DTB_NAME = value` enumerator of include/dtb.h."""
    src = open(os.path.join(ROOT, "include", "dtb.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return {k: int(v) for k, v in re.findall(r"\b(DTB_[A-Z0-9_]+)\s*=\s*(\d+)", src)}


def test_python_binding_constants_match_the_header():
    c = declared_constants()
    assert c["DTB_HOST"] == _lib.DTB_HOST and c["DTB_DEVICE"] == _lib.DTB_DEVICE
    for mode in ("AUTO", "PUSH", "PULL"):
        assert c[f"DTB_MODE_{mode}"] == getattr(_lib, f"MODE_{mode}")
    fields = {k[len("DTB_FIELD_"):]: v for k, v in c.items() if k.startswith("DTB_FIELD_")}
    tunes = {k[len("DTB_TUNE_"):]: v for k, v in c.items() if k.startswith("DTB_TUNE_")}
    assert fields and tunes
    for name, value in fields.items():
        assert getattr(_lib, f"FIELD_{name}") == value, name
    for name, value in tunes.items():
        assert getattr(_lib, f"TUNE_{name}") == value, name
    errors = {v for k, v in c.items() if k.startswith("DTB_ERR_")} | {c["DTB_OK"]}
    assert errors == set(_lib.STATUS)
