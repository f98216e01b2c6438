"""dtb_step_preallocated: one time step of a network whose device arrays the
caller owns, with the library allocating nothing.

It exists for callers that cannot allocate device memory or let a library do
it: code running inside another framework that owns a fixed memory pool or
budget, or a real-time stepping loop in which cudaMalloc / cudaFree (and the
device-wide synchronisation they can cause) are not allowed.  Its scratch
memory is a fixed static device array inside libdtb.so.

The test builds the same network twice — once as a library-owned handle
(dtb_block_create_synthetic + dtb_block_run in pull mode, the existing entry
point) and once as plain caller-owned device tensors — and checks that calls in
a row of the allocation-free entry point give the same V, J, t_last and
per-subblock results, bit for bit (the pull path's tolerance is zero): the first
two calls, and then enough calls (100) that the neurons leave the 5 ms (50-step)
refractory window every neuron starts in, so threshold crossings, t_last and
spike propagation are compared too.  Variants: isolated steps, no statistics
outputs (the scratch's spare rows), no subblocks.  The device's free memory must
not change across the calls after the first.  It also checks that sizes beyond
the fixed scratch are rejected.  The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest
import torch

from digital_twin_brain_b200 import Network, _lib, synthetic
from digital_twin_brain_b200._lib import FIELD_J, FIELD_T_LAST, FIELD_V
from tests._helpers import decay_like_reference

pytestmark = pytest.mark.gpu

DTB_ERR_LIMIT = 7
MAX_NEURONS = 1 << 22
MAX_SUBBLOCKS = 1024


class PreallocNet(ctypes.Structure):
    _fields_ = [("n_neurons", ctypes.c_int64), ("n_subblocks", ctypes.c_int32), ("device", ctypes.c_int32),
                ("V", ctypes.c_void_p), ("J", ctypes.c_void_p), ("t_last", ctypes.c_void_p),
                ("cls", ctypes.c_void_p), ("classes", ctypes.c_void_p), ("sub_count", ctypes.c_void_p),
                ("rowptr", ctypes.c_void_p),
                ("index", ctypes.c_void_p), ("weight", ctypes.c_void_p), ("dt", ctypes.c_float),
                ("seed", ctypes.c_uint64), ("stream_id", ctypes.c_uint32)]


CLASS_DTYPE = np.dtype([("g", "<f4", 4), ("V_ui", "<f4", 4), ("decay", "<f4", 4), ("g_L", "<f4"), ("V_L", "<f4"),
                        ("rC_dt", "<f4"), ("V_th", "<f4"), ("V_reset", "<f4"), ("T_ref", "<f4"),
                        ("I_ext", "<f4"), ("noise_rate", "<f4"), ("subblock", "<i4"), ("C", "<f4"),
                        ("pad0", "<f4"), ("pad1", "<f4")])


def class_table(spec, class_decay):
    """dtb_param_class rows for the spec's classes (subblock = class index)."""
    assert CLASS_DTYPE.itemsize == 96
    cp = spec.class_property
    t = np.zeros(len(cp), CLASS_DTYPE)
    t["g"], t["V_ui"], t["decay"] = cp[:, 10:14], cp[:, 14:18], class_decay
    t["g_L"], t["V_L"], t["V_th"], t["V_reset"] = cp[:, 6], cp[:, 7], cp[:, 8], cp[:, 9]
    t["rC_dt"] = (np.float32(1.0) / cp[:, 4]) * np.float32(spec.dt)       # C.reciprocal() * dt in float32
    t["T_ref"], t["I_ext"], t["noise_rate"], t["C"] = cp[:, 5], cp[:, 2], cp[:, 0], cp[:, 4]
    t["subblock"] = np.arange(len(cp))
    return t


def per_class_decay(spec):
    d = decay_like_reference(spec.property(), spec.dt).T
    cls = spec.neuron_class()
    return np.stack([d[np.argmax(cls == c)] for c in range(2 * spec.R)])


def step_fn():
    # a separate handle of the library, so these argtypes stay local to this test
    fn = ctypes.CDLL(_lib.lib_path()).dtb_step_preallocated
    fn.argtypes = [ctypes.POINTER(PreallocNet), ctypes.c_float, ctypes.c_uint64, ctypes.c_float, ctypes.c_int,
                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return fn


@pytest.mark.parametrize("case", ["plain", "isolated", "no_outputs", "no_subblocks"])
def test_preallocated_step_matches_library_owned_run(case):
    spec = synthetic.single_block(20000, 100, name="prealloc_20k")
    cdec = per_class_decay(spec)
    ref = Network.from_spec(spec, device=0, build_push=False, class_decay=cdec)

    # caller-owned copy of the same network on the device
    dev = torch.device("cuda", 0)
    rowptr, index, weight = ref.get_csr("pull")
    cp = spec.class_property
    cls_np = spec.neuron_class()
    v0 = ((cp[cls_np, 8] + cp[cls_np, 9]) / np.float32(2)).astype(np.float32)   # models/block.py:56
    V = torch.from_numpy(v0).to(dev)
    J = torch.zeros((spec.N, 4), dtype=torch.float32, device=dev)
    t_last = torch.zeros(spec.N, dtype=torch.float32, device=dev)
    cls = torch.from_numpy(cls_np.astype(np.int32)).to(dev)
    classes = torch.from_numpy(class_table(spec, cdec).view(np.uint8)).to(dev)
    rp = torch.from_numpy(rowptr).to(dev)
    ix = torch.from_numpy(index.view(np.int32)).to(dev)
    w = torch.from_numpy(weight).to(dev)
    n_sub = 0 if case == "no_subblocks" else 2 * spec.R
    sub_count = torch.from_numpy(np.bincount(cls_np, minlength=2 * spec.R).astype(np.int32)).to(dev)
    sums = torch.empty(2 * spec.R, dtype=torch.float32, device=dev)
    means = torch.empty(2 * spec.R, dtype=torch.float32, device=dev)
    outputs = case in ("plain", "isolated")
    net = PreallocNet(n_neurons=spec.N, n_subblocks=n_sub, device=0, V=V.data_ptr(), J=J.data_ptr(),
                      t_last=t_last.data_ptr(), cls=cls.data_ptr(), classes=classes.data_ptr(),
                      sub_count=sub_count.data_ptr() if n_sub else None, rowptr=rp.data_ptr(), index=ix.data_ptr(),
                      weight=w.data_ptr(), dt=spec.dt, seed=spec.seed, stream_id=spec.stream_id)
    fn = step_fn()
    stream = torch.cuda.current_stream(dev)
    t = np.float32(0.0)
    iso = case == "isolated"
    spiked = 0
    for step in range(100):
        stream.synchronize()
        free_before = torch.cuda.mem_get_info(dev)[0]
        rc = fn(ctypes.byref(net), float(t), step, 0.01, int(iso), sums.data_ptr() if outputs else None,
                means.data_ptr() if outputs else None, ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0
        stream.synchronize()
        if step > 0:   # the calls after the first allocate nothing on the device
            assert torch.cuda.mem_get_info(dev)[0] == free_before
        t = np.float32(t + np.float32(spec.dt))
        s_ref, m_ref, _ = ref.run(1, noise_rate=0.01, isolated=iso, mode="pull")
        spiked += int(s_ref[0].sum())
        if outputs:
            assert np.array_equal(sums.cpu().numpy(), s_ref[0])
            assert np.array_equal(means.cpu().numpy(), m_ref[0])
        if step < 2 or step % 10 == 9:
            assert np.array_equal(V.cpu().numpy(), ref.get(FIELD_V)), f"V differs after call {step + 1}"
            assert np.array_equal(J.cpu().numpy().T, ref.get(FIELD_J)), f"J differs after call {step + 1}"
            assert np.array_equal(t_last.cpu().numpy(), ref.get(FIELD_T_LAST))
    assert float(t) == np.float32(ref.get(7))  # block.t advances identically
    assert spiked > 0                          # threshold crossings after the refractory window
    assert (t_last.cpu().numpy() > 0).any()


def test_preallocated_step_rejects_sizes_beyond_its_scratch():
    fn = step_fn()
    dummy = torch.zeros(16, dtype=torch.float32, device="cuda:0")
    p = dummy.data_ptr()
    big = PreallocNet(n_neurons=MAX_NEURONS + 1, n_subblocks=2, device=0, V=p, J=p, t_last=p, cls=p, classes=p,
                      sub_count=p, rowptr=p, index=p, weight=p, dt=0.1, seed=0, stream_id=0)
    assert fn(ctypes.byref(big), 0.0, 0, 0.01, 0, None, None, None) == DTB_ERR_LIMIT
    many = PreallocNet(n_neurons=16, n_subblocks=MAX_SUBBLOCKS + 1, device=0, V=p, J=p, t_last=p, cls=p,
                       classes=p, sub_count=p, rowptr=p, index=p, weight=p, dt=0.1, seed=0, stream_id=0)
    assert fn(ctypes.byref(many), 0.0, 0, 0.01, 0, None, None, None) == DTB_ERR_LIMIT
