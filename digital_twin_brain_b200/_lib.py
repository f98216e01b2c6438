"""ctypes binding of libdtb.so (include/dtb.h).

The library must have been built (``digital_twin_brain_b200.build``); there is
no fallback: every entry point fails loudly when the CUDA library is missing.
"""
from __future__ import annotations

import ctypes
import os
import threading

from . import build as _build

c_int, c_i64, c_u64, c_u32, c_f32, c_f64 = (ctypes.c_int, ctypes.c_int64, ctypes.c_uint64, ctypes.c_uint32,
                                            ctypes.c_float, ctypes.c_double)
c_vp, c_char_p, c_size_t = ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t

DTB_HOST, DTB_DEVICE = 0, 1
MODE_AUTO, MODE_PUSH, MODE_PULL = 0, 1, 2
MODES = {"auto": MODE_AUTO, "push": MODE_PUSH, "pull": MODE_PULL}

FIELD_V, FIELD_J, FIELD_I_UI, FIELD_I_SYN, FIELD_T_LAST, FIELD_ACTIVE, FIELD_NEW_ACTIVE, FIELD_T, FIELD_STEP, \
    FIELD_SUB_COUNT, FIELD_EVENTS, FIELD_WINDOW_SPIKES, FIELD_G_FACTOR = range(13)

TUNE_SCATTER_WORDS, TUNE_CHUNK, TUNE_PULL_THRESHOLD_PPM, TUNE_USE_GRAPHS, TUNE_STEP_VARIANT, TUNE_PULL_METHOD, \
    TUNE_J_CACHE, TUNE_SCATTER_VARIANT, TUNE_PUSH_METHOD, TUNE_BIN_WORDS, TUNE_BIN_CAPACITY, TUNE_BIN_SHIFT, \
    TUNE_STAGE_WAIT_LIMIT, TUNE_SCATTER_REVERSE = range(14)

STATUS = {0: "ok", 1: "bad argument", 2: "CUDA error", 3: "out of memory", 4: "I/O error", 5: "format error",
          6: "invalid state", 7: "limit exceeded"}


class DtbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"dtb error {code} ({STATUS.get(code, '?')}): {msg}")
        self.code = code


class BlockDesc(ctypes.Structure):
    _fields_ = [("n_neurons", c_i64), ("property", c_vp), ("decay", c_vp), ("n_synapses", c_i64),
                ("post", c_vp), ("pre", c_vp), ("kind", c_vp), ("weight", c_vp), ("dt", c_f32),
                ("seed", c_u64), ("stream_id", c_u32), ("device", c_int), ("build_push", c_int)]


class SynthDesc(ctypes.Structure):
    _fields_ = [("n_regions", c_int), ("region_start", c_vp), ("region_n_exc", c_vp), ("cum", c_vp),
                ("K", c_int), ("w_scale", c_f32), ("gen_seed", c_u64), ("class_property", c_vp),
                ("class_decay", c_vp), ("dt", c_f32), ("seed", c_u64), ("stream_id", c_u32), ("device", c_int),
                ("build_push", c_int), ("src_base", c_vp), ("src_count", c_vp), ("cum_off", c_vp), ("cum_flat", c_vp),
                ("n_members", ctypes.c_int32), ("region_member", c_vp), ("member_start", c_vp),
                ("member_seed", c_vp)]


class BlockInfo(ctypes.Structure):
    _fields_ = [("n_neurons", c_i64), ("n_synapses", c_i64), ("n_subblocks", ctypes.c_int32),
                ("n_classes", ctypes.c_int32), ("has_pull", ctypes.c_int32), ("has_push", ctypes.c_int32),
                ("device_bytes", c_i64), ("max_outdegree", c_i64), ("max_indegree", c_i64),
                ("kernel_launches", c_i64)]


# name -> (argtypes)
_SIGS = {
    "dtb_abi_version": [],
    "dtb_last_error": [c_char_p, c_size_t],
    "dtb_block_create": [ctypes.POINTER(BlockDesc), ctypes.POINTER(c_vp)],
    "dtb_block_create_synthetic": [ctypes.POINTER(SynthDesc), ctypes.POINTER(c_vp)],
    "dtb_block_create_from_npz": [c_char_p, c_f32, c_u64, c_u32, c_int, c_int, ctypes.POINTER(c_vp)],
    "dtb_block_destroy": [c_vp],
    "dtb_block_set_stream": [c_vp, c_vp],
    "dtb_block_synchronize": [c_vp],
    "dtb_block_get_info": [c_vp, ctypes.POINTER(BlockInfo)],
    "dtb_block_run": [c_vp, c_int, c_f32, c_int, c_int, c_vp, c_vp, c_vp, c_int],
    "dtb_block_step_forced": [c_vp, c_f32, c_int, c_int, c_vp, c_vp, c_vp, c_vp, c_int],
    "dtb_block_time_kernels": [c_vp, c_int, c_f32, c_int, c_int, c_vp],
    "dtb_block_set_tuning": [c_vp, c_int, c_i64],
    "dtb_block_get_tuning": [c_vp, c_int, ctypes.POINTER(c_i64)],
    "dtb_block_autotune": [c_vp, c_int, c_f32, c_vp],
    "dtb_block_get": [c_vp, c_int, c_vp, c_int],
    "dtb_block_set": [c_vp, c_int, c_vp, c_int],
    "dtb_block_get_csr": [c_vp, c_int, c_vp, c_vp, c_vp, c_int],
    "dtb_block_get_csr_entries": [c_vp, c_int, c_i64, c_i64, c_vp, c_vp, c_int],
    "dtb_block_update_property": [c_vp, c_vp, c_vp],
    "dtb_block_scale_property_by_subblock": [c_vp, c_int, c_vp, c_vp, c_vp],
    "dtb_block_gamma_property_by_subblock": [c_vp, c_int, c_vp, c_vp, c_vp, c_vp],
    "dtb_block_set_input_spikes": [c_vp, c_i64, c_vp, c_i64, c_vp],
    "dtb_block_update_conn_weight": [c_vp, c_i64, c_vp, c_vp, c_vp, c_vp],
    "dtb_block_save": [c_vp, c_char_p],
    "dtb_block_load": [c_vp, c_char_p],
    "dtb_bold_create": [c_i64, c_int, c_f64, c_f64, c_f64, c_f64, c_f64, c_f64, c_f64, c_f64, c_int,
                        ctypes.POINTER(c_vp)],
    "dtb_bold_destroy": [c_vp],
    "dtb_bold_set_stream": [c_vp, c_vp],
    "dtb_bold_run": [c_vp, c_vp, c_vp, c_int],
    "dtb_bold_state_update": [c_vp, c_vp, c_i64, c_i64, c_i64, c_int],
    "dtb_bold_run_steps": [c_vp, c_vp, c_int, c_f64, c_vp, c_int],
    "dtb_bold_get": [c_vp, c_int, c_vp, c_int],
    "dtb_bold_set": [c_vp, c_int, c_vp, c_int],
    "dtb_block_attach_bold": [c_vp, c_int, c_vp, c_f64, c_f64, c_f64, c_f64, c_f64, c_f64, c_f64, c_f64],
    "dtb_block_get_bold": [c_vp, c_int, c_vp, c_int],
    "dtb_block_set_bold": [c_vp, c_int, c_vp, c_int],
    "dtb_block_set_samples": [c_vp, c_int, c_vp, c_i64],
    "dtb_block_get_samples": [c_vp, c_vp, c_vp, ctypes.POINTER(c_i64), c_int],
    "dtb_step_preallocated": [c_vp, c_f32, c_u64, c_f32, c_int, c_vp, c_vp, c_vp],
    "dtb_mlp_create": [c_int, c_int, c_u64, c_int, ctypes.POINTER(c_vp)],
    "dtb_mlp_destroy": [c_vp],
    "dtb_mlp_set_stream": [c_vp, c_vp],
    "dtb_mlp_n_params": [c_vp, ctypes.POINTER(c_i64)],
    "dtb_mlp_get_params": [c_vp, c_vp, c_int],
    "dtb_mlp_set_params": [c_vp, c_vp, c_int],
    "dtb_mlp_forward": [c_vp, c_vp, c_i64, c_vp],
    "dtb_mlp_gradient": [c_vp, c_vp, c_vp, c_i64, c_vp, c_vp],
    "dtb_mlp_train_step": [c_vp, c_vp, c_vp, c_i64, c_f32, c_vp],
    "dtb_mlp_last_error": [c_char_p, c_size_t],
}

_lock = threading.Lock()
_lib = None


def lib_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = True):
    """Load libdtb.so (building it first when absent and nvcc exists)."""
    global _lib
    with _lock:
        if _lib is None:
            path = _build.LIB
            if not os.path.exists(path):
                if not build_if_missing:
                    raise ImportError(f"{path} is missing; run python -m digital_twin_brain_b200.build")
                _build.build()
            L = ctypes.CDLL(path)
            for name, args in _SIGS.items():
                fn = getattr(L, name)
                fn.argtypes = args
                fn.restype = c_int
            _lib = L
    return _lib


def last_error() -> str:
    buf = ctypes.create_string_buffer(2048)
    load().dtb_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc: int, mlp: bool = False):
    if rc != 0:
        if mlp:
            buf = ctypes.create_string_buffer(1024)
            load().dtb_mlp_last_error(buf, len(buf))
            raise DtbError(rc, buf.value.decode(errors="replace"))
        raise DtbError(rc, last_error())


def call(name: str, *args):
    check(getattr(load(), name)(*args), mlp=name.startswith("dtb_mlp_"))
