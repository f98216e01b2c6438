"""Python handle over the C ABI: one network resident on one GPU.

This is the layer the drop-in classes (``models/block.py``,
``models/bold_model_pytorch.py``) and ``bench.py`` use.  Host arrays are
numpy; device arrays are torch CUDA tensors (torch is only the allocator).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import (DTB_DEVICE, DTB_HOST, FIELD_ACTIVE, FIELD_EVENTS, FIELD_I_SYN, FIELD_I_UI, FIELD_J,
                   FIELD_G_FACTOR, FIELD_NEW_ACTIVE, FIELD_STEP, FIELD_SUB_COUNT, FIELD_T, FIELD_T_LAST, FIELD_V,
                   FIELD_WINDOW_SPIKES,
                   MODES)
from .synthetic import NetworkSpec

_FIELD_SHAPE = {FIELD_V: (1, np.float32), FIELD_J: (4, np.float32), FIELD_I_UI: (4, np.float32),
                FIELD_I_SYN: (1, np.float32), FIELD_T_LAST: (1, np.float32), FIELD_ACTIVE: (1, np.uint8),
                FIELD_NEW_ACTIVE: (1, np.uint8)}
_TORCH = {np.float32: torch.float32, np.uint8: torch.uint8, np.float64: torch.float64, np.uint32: torch.int32}


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, torch.Tensor):
        return ctypes.c_void_p(a.data_ptr())
    return a.ctypes.data_as(ctypes.c_void_p)


class Network:
    """A network of LIF neurons on one CUDA device (handle of ``dtb_block``)."""

    def __init__(self, handle: ctypes.c_void_p, device: int, dt: float):
        self._h = handle
        self.device = int(device)
        self.dt = float(dt)
        info = self.info()
        self.N = int(info.n_neurons)
        self.S = int(info.n_synapses)
        self.n_sub = int(info.n_subblocks)

    # ------------------------------------------------------------ creation
    @classmethod
    def from_arrays(cls, property: np.ndarray, post, pre, kind, weight, dt: float, seed: int = 0,
                    decay: np.ndarray | None = None, device: int = 0, build_push: bool = True,
                    stream_id: int = 0) -> "Network":
        """models/block.py:30 block(...) from host arrays: property [N,22], synapses (post, pre,
        kind in {0,2}, weight [S,2]) in the order sparse.mm accumulates them."""
        prop = np.ascontiguousarray(property, np.float32)
        N = prop.shape[0]
        post = np.ascontiguousarray(post, np.uint32)
        pre = np.ascontiguousarray(pre, np.uint32)
        kind = np.ascontiguousarray(kind, np.uint8)
        w = np.ascontiguousarray(weight, np.float32).reshape(-1, 2)
        dec = None if decay is None else np.ascontiguousarray(decay, np.float32).reshape(N, 4)
        d = _lib.BlockDesc(n_neurons=N, property=_ptr(prop), decay=_ptr(dec), n_synapses=len(post),
                           post=_ptr(post), pre=_ptr(pre), kind=_ptr(kind), weight=_ptr(w), dt=float(dt),
                           seed=int(seed), stream_id=int(stream_id), device=int(device),
                           build_push=int(bool(build_push)))
        h = ctypes.c_void_p()
        _lib.call("dtb_block_create", ctypes.byref(d), ctypes.byref(h))
        return cls(h, device, dt)

    @classmethod
    def from_spec(cls, spec: NetworkSpec, device: int = 0, build_push: bool = True,
                  class_decay: np.ndarray | None = None) -> "Network":
        """Generate a synthetic network on the device (identical to oracle.gen_network)."""
        rs = np.ascontiguousarray(spec.region_start, np.int64)
        ne = np.ascontiguousarray(spec.region_n_exc, np.int64)
        cum = np.ascontiguousarray(spec.cum, np.float32)
        cp = np.ascontiguousarray(spec.class_property, np.float32)
        cd = None if class_decay is None else np.ascontiguousarray(class_decay, np.float32)
        d = _lib.SynthDesc(n_regions=spec.R, region_start=_ptr(rs), region_n_exc=_ptr(ne), cum=_ptr(cum), K=spec.K,
                           w_scale=float(spec.w_scale), gen_seed=int(spec.gen_seed), class_property=_ptr(cp),
                           class_decay=_ptr(cd), dt=float(spec.dt), seed=int(spec.seed),
                           stream_id=int(spec.stream_id), device=int(device), build_push=int(bool(build_push)))
        keep = []
        if spec.members is not None:
            t = spec.members
            arrs = dict(src_base=np.ascontiguousarray(t["src_base"], np.int32),
                        src_count=np.ascontiguousarray(t["src_count"], np.int32),
                        cum_off=np.ascontiguousarray(t["cum_off"], np.int64),
                        cum_flat=np.ascontiguousarray(t["cum_flat"], np.float32),
                        region_member=np.ascontiguousarray(t["region_member"], np.int32),
                        member_start=np.ascontiguousarray(t["member_start"], np.int64),
                        member_seed=np.ascontiguousarray(t["member_seed"], np.uint64))
            keep.append(arrs)
            for k, v in arrs.items():
                setattr(d, k, _ptr(v))
            d.n_members = len(arrs["member_start"])
        h = ctypes.c_void_p()
        _lib.call("dtb_block_create_synthetic", ctypes.byref(d), ctypes.byref(h))
        return cls(h, device, spec.dt)

    @classmethod
    def from_npz(cls, directory: str, dt: float, seed: int = 0, device: int = 0, build_push: bool = True,
                 stream_id: int = 0) -> "Network":
        """generation/read_block.py:12 connect_for_block(directory) on the device."""
        h = ctypes.c_void_p()
        _lib.call("dtb_block_create_from_npz", directory.encode(), float(dt), int(seed), int(stream_id),
                  int(device), int(bool(build_push)), ctypes.byref(h))
        return cls(h, device, dt)

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().dtb_block_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------ info
    def info(self) -> _lib.BlockInfo:
        inf = _lib.BlockInfo()
        _lib.call("dtb_block_get_info", self._h, ctypes.byref(inf))
        return inf

    def synchronize(self):
        _lib.call("dtb_block_synchronize", self._h)

    def _torch_ready(self):
        """Before the library writes into (or reads) torch device memory on its own stream: torch's
        caching allocator may have handed out memory that work still queued on torch's current
        stream uses, so that work must finish first."""
        torch.cuda.current_stream(self.device).synchronize()

    # ------------------------------------------------------------ stepping
    def run(self, n_steps: int, noise_rate: float | None = 0.01, isolated: bool = False, mode: str = "auto",
            out: str = "host"):
        """n_steps x block.run; returns per-step (spike sums [n,n_sub], mean V [n,n_sub], propagated count [n]).
        noise_rate None selects the per-neuron rate of property column 0.  out: 'host' (numpy),
        'device' (torch CUDA tensors) or None (nothing returned, no host synchronisation)."""
        rate = -1.0 if noise_rate is None else float(noise_rate)
        m = MODES[mode]
        if out is None:
            _lib.call("dtb_block_run", self._h, int(n_steps), rate, int(bool(isolated)), m, None, None, None,
                      DTB_DEVICE)
            return None
        if out == "device":
            dev = torch.device("cuda", self.device)
            s = torch.empty((n_steps, self.n_sub), dtype=torch.float32, device=dev)
            mn = torch.empty((n_steps, self.n_sub), dtype=torch.float32, device=dev)
            na = torch.empty((n_steps,), dtype=torch.int32, device=dev)
            self._torch_ready()
            _lib.call("dtb_block_run", self._h, int(n_steps), rate, int(bool(isolated)), m, _ptr(s), _ptr(mn),
                      _ptr(na), DTB_DEVICE)
            self.synchronize()
            return s, mn, na
        s = np.empty((n_steps, self.n_sub), np.float32)
        mn = np.empty((n_steps, self.n_sub), np.float32)
        na = np.empty((n_steps,), np.uint32)
        _lib.call("dtb_block_run", self._h, int(n_steps), rate, int(bool(isolated)), m, _ptr(s), _ptr(mn), _ptr(na),
                  DTB_HOST)
        return s, mn, na

    def set_stream(self, stream):
        """Issue all of this network's work on `stream` (a torch.cuda.Stream or a raw cudaStream_t int)."""
        raw = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)
        _lib.call("dtb_block_set_stream", self._h, ctypes.c_void_p(raw))

    def time_kernels(self, n_steps: int, noise_rate: float | None = 0.01, isolated: bool = False,
                     mode: str = "auto") -> dict:
        """Per-kernel CUDA-event timing of n_steps (no graphs)."""
        out = np.zeros(4, np.float32)
        rate = -1.0 if noise_rate is None else float(noise_rate)
        _lib.call("dtb_block_time_kernels", self._h, int(n_steps), rate, int(bool(isolated)), MODES[mode], _ptr(out))
        return dict(update_ms=float(out[0]), propagate_ms=float(out[1]), step_ms=float(out[2]),
                    events_per_step=float(out[3]))

    def set_tuning(self, key: int, value: int):
        _lib.call("dtb_block_set_tuning", self._h, int(key), int(value))

    def get_tuning(self, key: int) -> int:
        v = ctypes.c_int64()
        _lib.call("dtb_block_get_tuning", self._h, int(key), ctypes.byref(v))
        return int(v.value)

    def autotune(self, n_steps: int = 32, noise_rate: float = 0.01) -> dict:
        """Pick the scatter launch shape and the push/pull threshold by measurement (advances the run)."""
        r = np.zeros(6, np.float32)
        _lib.call("dtb_block_autotune", self._h, int(n_steps), float(noise_rate), _ptr(r))
        return dict(scatter_words=int(r[0]), push_ms=float(r[1]), pull_ms=float(r[2]), activity=float(r[3]),
                    pull_threshold=float(r[4]), step_variant=int(r[5]),
                    j_cache=self.get_tuning(_lib.TUNE_J_CACHE),
                    scatter_variant=self.get_tuning(_lib.TUNE_SCATTER_VARIANT),
                    scatter_reverse=self.get_tuning(_lib.TUNE_SCATTER_REVERSE),
                    push_method=self.get_tuning(_lib.TUNE_PUSH_METHOD))

    def step_forced(self, forced_active=None, forced_new_active=None, noise_rate: float | None = 0.01,
                    isolated: bool = False, mode: str = "pull"):
        """One step with this step's active / new_active sets replaced (teacher forcing)."""
        fa = None if forced_active is None else np.ascontiguousarray(forced_active, np.uint8)
        fn = None if forced_new_active is None else np.ascontiguousarray(forced_new_active, np.uint8)
        s = np.empty(self.n_sub, np.float32)
        mn = np.empty(self.n_sub, np.float32)
        rate = -1.0 if noise_rate is None else float(noise_rate)
        _lib.call("dtb_block_step_forced", self._h, rate, int(bool(isolated)), MODES[mode], _ptr(fa), _ptr(fn),
                  _ptr(s), _ptr(mn), DTB_HOST)
        return s, mn

    # ------------------------------------------------------------ state
    def get(self, field: int, device: bool = False):
        """State array (numpy on the host, or a torch CUDA tensor with device=True)."""
        if field in (FIELD_T,):
            out = np.zeros(1, np.float32)
            _lib.call("dtb_block_get", self._h, field, _ptr(out), DTB_HOST)
            return float(out[0])
        if field in (FIELD_STEP, FIELD_EVENTS):
            out = np.zeros(1, np.uint64)
            _lib.call("dtb_block_get", self._h, field, _ptr(out), DTB_HOST)
            return int(out[0])
        if field == FIELD_SUB_COUNT:
            out = np.zeros(self.n_sub, np.uint32)
            _lib.call("dtb_block_get", self._h, field, _ptr(out), DTB_HOST)
            return out
        rows, dt = _FIELD_SHAPE[field]
        shape = (rows, self.N) if rows > 1 else (self.N,)
        if device:
            out = torch.empty(shape, dtype=_TORCH[dt], device=torch.device("cuda", self.device))
            self._torch_ready()
            _lib.call("dtb_block_get", self._h, field, _ptr(out), DTB_DEVICE)
            self.synchronize()
            return out
        out = np.empty(shape, dt)
        _lib.call("dtb_block_get", self._h, field, _ptr(out), DTB_HOST)
        return out

    def get_csr(self, which: str = "pull"):
        """(rowptr [N+1] int64, index [S] uint32 with bit 31 = GABA pair, weight [S,2] float32) on the host."""
        rp = np.empty(self.N + 1, np.int64)
        ix = np.empty(self.S, np.uint32)
        w = np.empty((self.S, 2), np.float32)
        _lib.call("dtb_block_get_csr", self._h, 0 if which == "pull" else 1, _ptr(rp), _ptr(ix), _ptr(w), DTB_HOST)
        return rp, ix, w

    def get_csr_rowptr(self, which: str = "pull") -> np.ndarray:
        rp = np.empty(self.N + 1, np.int64)
        _lib.call("dtb_block_get_csr", self._h, 0 if which == "pull" else 1, _ptr(rp), None, None, DTB_HOST)
        return rp

    def get_csr_entries(self, which: str, first: int, count: int, device: bool = False, weights: bool = True):
        """Entries [first, first+count) of a CSR: (index uint32 with bit 31 = GABA pair, weight [count,2]);
        numpy on the host, or torch CUDA tensors (index as int32 bits) with device=True."""
        which_i = 0 if which == "pull" else 1
        if device:
            dev = torch.device("cuda", self.device)
            ix = torch.empty(count, dtype=torch.int32, device=dev)
            w = torch.empty((count, 2), dtype=torch.float32, device=dev) if weights else None
            self._torch_ready()
            _lib.call("dtb_block_get_csr_entries", self._h, which_i, int(first), int(count), _ptr(ix), _ptr(w),
                      DTB_DEVICE)
            self.synchronize()
            return ix, w
        ix = np.empty(count, np.uint32)
        w = np.empty((count, 2), np.float32) if weights else None
        _lib.call("dtb_block_get_csr_entries", self._h, which_i, int(first), int(count), _ptr(ix), _ptr(w), DTB_HOST)
        return ix, w

    def set(self, field: int, value):
        if field == FIELD_T:
            arr = np.asarray([value], np.float32)
        elif field == FIELD_STEP:
            arr = np.asarray([value], np.uint64)
        else:
            arr = np.ascontiguousarray(value, np.float32)
        _lib.call("dtb_block_set", self._h, field, _ptr(arr), DTB_HOST)

    def update_property(self, property: np.ndarray, decay: np.ndarray | None = None):
        prop = np.ascontiguousarray(property, np.float32)
        dec = None if decay is None else np.ascontiguousarray(decay, np.float32)
        _lib.call("dtb_block_update_property", self._h, _ptr(prop), _ptr(dec))

    def scale_property_by_subblock(self, sub, col, value):
        sub = np.ascontiguousarray(sub, np.int32)
        col = np.ascontiguousarray(col, np.int32)
        value = np.ascontiguousarray(value, np.float32)
        _lib.call("dtb_block_scale_property_by_subblock", self._h, len(sub), _ptr(sub), _ptr(col), _ptr(value))

    def set_input_spikes(self, neurons, spikes):
        """Input neurons replaying a raster spikes[i, t] (models/block.py:37-50, :104-109); T columns serve
        T - 1 steps.  neurons=[] removes them."""
        idx = np.ascontiguousarray(neurons, np.uint32)
        if len(idx) == 0:
            _lib.call("dtb_block_set_input_spikes", self._h, 0, None, 0, None)
            return
        sp = np.ascontiguousarray(spikes, np.uint8)
        assert sp.ndim == 2 and sp.shape[0] == len(idx)
        _lib.call("dtb_block_set_input_spikes", self._h, len(idx), _ptr(idx), sp.shape[1], _ptr(sp))

    def gamma_property_by_subblock(self, sub, col, alpha, beta):
        """Column col[i] of every neuron of subblock sub[i] <- Gamma(alpha[i], 1) / beta[i] per neuron
        (cuda/src/stage/property.cpp:313-471); g_ui columns per neuron, others in the delta limit."""
        sub = np.ascontiguousarray(sub, np.int32)
        col = np.ascontiguousarray(col, np.int32)
        a = np.ascontiguousarray(alpha, np.float32)
        b = np.ascontiguousarray(beta, np.float32)
        _lib.call("dtb_block_gamma_property_by_subblock", self._h, len(sub), _ptr(sub), _ptr(col), _ptr(a), _ptr(b))

    def g_factors(self) -> np.ndarray:
        """Per-neuron g_ui factors [N, 4] set by gamma_property_by_subblock."""
        out = np.empty((self.N, 4), np.float32)
        _lib.call("dtb_block_get", self._h, FIELD_G_FACTOR, _ptr(out), DTB_HOST)
        return out

    def update_conn_weight(self, channel, post, pre, value):
        ch = np.ascontiguousarray(channel, np.uint8)
        po = np.ascontiguousarray(post, np.uint32)
        pr = np.ascontiguousarray(pre, np.uint32)
        v = np.ascontiguousarray(value, np.float32)
        _lib.call("dtb_block_update_conn_weight", self._h, len(ch), _ptr(ch), _ptr(po), _ptr(pr), _ptr(v))

    def save(self, path: str):
        _lib.call("dtb_block_save", self._h, str(path).encode())

    def load(self, path: str):
        _lib.call("dtb_block_load", self._h, str(path).encode())

    # ------------------------------------------------------------ BOLD
    def attach_bold(self, sub_to_region, n_regions: int, epsilon=200, tao_s=0.8, tao_f=0.4, tao_0=1, alpha=0.2,
                    E_0=0.8, V_0=0.02, delta_t: float | None = None):
        """simulation/simulation.py:269-279 per step; delta_t defaults to dt / 1000 (seconds per step)."""
        s2r = np.ascontiguousarray(sub_to_region, np.int32)
        dts = self.dt / 1000.0 if delta_t is None else float(delta_t)
        _lib.call("dtb_block_attach_bold", self._h, int(n_regions), _ptr(s2r), float(epsilon), float(tao_s),
                  float(tao_f), float(tao_0), float(alpha), float(E_0), float(V_0), dts)
        self.n_regions = int(n_regions)

    def get_bold(self, field: str = "bold", device: bool = False):
        idx = {"s": 0, "q": 1, "v": 2, "f_in": 3, "bold": 4, "act": 5}[field]
        if device:
            out = torch.empty(self.n_regions, dtype=torch.float64, device=torch.device("cuda", self.device))
            self._torch_ready()
            _lib.call("dtb_block_get_bold", self._h, idx, _ptr(out), DTB_DEVICE)
            self.synchronize()
            return out
        out = np.empty(self.n_regions, np.float64)
        _lib.call("dtb_block_get_bold", self._h, idx, _ptr(out), DTB_HOST)
        return out

    def set_bold(self, field: str, value):
        """Overwrite the BOLD state s, q, v or f_in (host array or CUDA tensor of n_regions doubles)."""
        idx = {"s": 0, "q": 1, "v": 2, "f_in": 3}[field]
        if isinstance(value, torch.Tensor) and value.is_cuda:
            v = value.to(torch.float64).contiguous()
            torch.cuda.current_stream(self.device).synchronize()
            _lib.call("dtb_block_set_bold", self._h, idx, _ptr(v), DTB_DEVICE)
        else:
            v = np.ascontiguousarray(value, np.float64)
            _lib.call("dtb_block_set_bold", self._h, idx, _ptr(v), DTB_HOST)

    def set_samples(self, idx, capacity_steps: int):
        """Record spike and V of neurons idx after every step (ring of capacity_steps rows)."""
        idx = np.ascontiguousarray(idx, np.uint32)
        self.n_samples = len(idx)
        _lib.call("dtb_block_set_samples", self._h, len(idx), _ptr(idx) if len(idx) else None, int(capacity_steps))

    def get_samples(self, out: str = "host"):
        """(spikes [rows, n] uint8, V [rows, n] float32), oldest step first; out 'host' (numpy) or 'device'
        (torch CUDA tensors)."""
        n = getattr(self, "n_samples", 0)
        rows = ctypes.c_int64()
        _lib.call("dtb_block_get_samples", self._h, None, None, ctypes.byref(rows), DTB_HOST)
        if out == "device":
            dev = torch.device("cuda", self.device)
            sp = torch.empty((rows.value, n), dtype=torch.uint8, device=dev)
            v = torch.empty((rows.value, n), dtype=torch.float32, device=dev)
            if rows.value and n:
                self._torch_ready()
                _lib.call("dtb_block_get_samples", self._h, _ptr(sp), _ptr(v), ctypes.byref(rows), DTB_DEVICE)
                self.synchronize()
            return sp, v
        sp = np.empty((rows.value, n), np.uint8)
        v = np.empty((rows.value, n), np.float32)
        if rows.value and n:
            _lib.call("dtb_block_get_samples", self._h, _ptr(sp), _ptr(v), ctypes.byref(rows), DTB_HOST)
        return sp, v

    def window_spikes(self) -> np.ndarray:
        """Spikes per subblock since the last clear_window_spikes() (uint64 [n_sub])."""
        out = np.empty(self.n_sub, np.uint64)
        _lib.call("dtb_block_get", self._h, FIELD_WINDOW_SPIKES, _ptr(out), DTB_HOST)
        return out

    def clear_window_spikes(self):
        z = np.zeros(self.n_sub, np.uint64)
        _lib.call("dtb_block_set", self._h, FIELD_WINDOW_SPIKES, _ptr(z), DTB_HOST)


class BoldModel:
    """Handle of ``dtb_bold`` (models/bold_model_pytorch.py on the device)."""

    def __init__(self, n_regions: int, dtype=torch.float32, epsilon=200, tao_s=0.8, tao_f=0.4, tao_0=1, alpha=0.2,
                 E_0=0.8, V_0=0.02, delta_t=1e-3, device: int = 0):
        self.R = int(n_regions)
        self.dtype = dtype
        self.device = int(device)
        h = ctypes.c_void_p()
        _lib.call("dtb_bold_create", self.R, 1 if dtype == torch.float64 else 0, float(epsilon), float(tao_s),
                  float(tao_f), float(tao_0), float(alpha), float(E_0), float(V_0), float(delta_t), self.device,
                  ctypes.byref(h))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().dtb_bold_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _dev(self, t: torch.Tensor) -> torch.Tensor:
        return t.to(device=torch.device("cuda", self.device), dtype=self.dtype).contiguous()

    def _on_torch_stream(self):
        # every call is ordered on torch's current stream of the model's device
        _lib.call("dtb_bold_set_stream", self._h,
                  ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream))

    def run(self, u: torch.Tensor) -> torch.Tensor:
        du = self._dev(u)
        out = torch.empty_like(du)
        self._on_torch_stream()
        _lib.call("dtb_bold_run", self._h, _ptr(du), _ptr(out), DTB_DEVICE)
        return out

    def run_steps(self, u: torch.Tensor, n_steps: int, u_floor: float = 1e-5) -> torch.Tensor:
        """n_steps BOLD steps with constant input max(u, u_floor); returns the last signal."""
        du = self._dev(u)
        out = torch.empty_like(du)
        self._on_torch_stream()
        _lib.call("dtb_bold_run_steps", self._h, _ptr(du), int(n_steps), float(u_floor), _ptr(out), DTB_DEVICE)
        return out

    def state_update(self, w: torch.Tensor):
        dw = self._dev(w)
        self._on_torch_stream()
        _lib.call("dtb_bold_state_update", self._h, _ptr(dw), dw.shape[0], dw.shape[1], dw.shape[2], DTB_DEVICE)

    def get(self, field: int) -> torch.Tensor:
        out = torch.empty(self.R, dtype=self.dtype, device=torch.device("cuda", self.device))
        self._on_torch_stream()
        _lib.call("dtb_bold_get", self._h, field, _ptr(out), DTB_DEVICE)
        return out

    def set(self, field: int, value: torch.Tensor):
        dv = self._dev(value).reshape(-1)
        if dv.numel() != self.R:
            raise ValueError(f"state of {dv.numel()} regions for a model of {self.R}")
        self._on_torch_stream()
        _lib.call("dtb_bold_set", self._h, field, _ptr(dv), DTB_DEVICE)
