"""Drop-in replacement of the reference's ``models/bold_model_pytorch.py`` ``BOLD``.

The Balloon-Windkessel Euler step (bold_model_pytorch.py:43-78) runs in a
CUDA kernel (libdtb ``dtb_bold_*``) in the dtype of the input (float32 or
float64), with the reference's update order (q, v, f_in, s) and clamps.
State tensors ``s``, ``q``, ``v``, ``f_in`` live on the GPU.
"""
from __future__ import annotations

import numpy as np
import torch

from ..network import BoldModel

_FIELDS = {"s": 0, "q": 1, "v": 2, "f_in": 3}


class BOLD:
    def __init__(self, epsilon, tao_s, tao_f, tao_0, alpha, E_0, V_0, delta_t=1e-3, init_f_in=None, init_s=None,
                 init_v=None, init_q=None, device: int | None = None):
        self.epsilon = epsilon
        self.tao_s = tao_s
        self.tao_f = tao_f
        self.tao_0 = tao_0
        self.E_0 = E_0
        self.V_0 = V_0
        self.delta_t = delta_t
        self.alpha = alpha
        self.div_alpha = 1 / alpha
        self._device = torch.cuda.current_device() if device is None else int(device)
        self._model: BoldModel | None = None
        self._pending = {"f_in": init_f_in, "s": init_s, "v": init_v, "q": init_q}

    def _ensure(self, n: int, dtype: torch.dtype):
        if self._model is not None and self._model.R == n and self._model.dtype == dtype:
            return
        self._model = BoldModel(n, dtype=dtype, epsilon=self.epsilon, tao_s=self.tao_s, tao_f=self.tao_f,
                                tao_0=self.tao_0, alpha=self.alpha, E_0=self.E_0, V_0=self.V_0,
                                delta_t=self.delta_t, device=self._device)
        for k, v in self._pending.items():
            if v is not None:
                self._model.set(_FIELDS[k], torch.as_tensor(v))
        self._pending = {k: None for k in self._pending}

    @staticmethod
    def _as_tensor(u):
        if isinstance(u, np.ndarray):  # bold_model_pytorch.py:58-59 promotes ndarrays to float64
            return torch.from_numpy(u.astype(np.float64))
        return u

    def state_update(self, w):
        """bold_model_pytorch.py:34-41."""
        w = self._as_tensor(w)
        dtype = torch.float64 if w.dtype == torch.float64 else torch.float32
        self._ensure(w.shape[0] * w.shape[1], dtype)
        self._model.state_update(w)

    def run(self, u):
        """bold_model_pytorch.py:43-78: one Euler step; returns the BOLD signal of every region."""
        u = self._as_tensor(u)
        dtype = torch.float64 if u.dtype == torch.float64 else torch.float32
        self._ensure(u.numel(), dtype)
        out = self._model.run(u.reshape(-1))
        return out.reshape(u.shape).to(u.device)

    def _get(self, name):
        if self._model is None:
            return self._pending[name]
        return self._model.get(_FIELDS[name])

    def _set(self, name, value):
        if self._model is None:
            self._pending[name] = value
        elif value is not None:
            self._model.set(_FIELDS[name], torch.as_tensor(value))

    s = property(lambda self: self._get("s"), lambda self, v: self._set("s", v))
    q = property(lambda self: self._get("q"), lambda self, v: self._set("q", v))
    v = property(lambda self: self._get("v"), lambda self, v: self._set("v", v))
    f_in = property(lambda self: self._get("f_in"), lambda self, v: self._set("f_in", v))
