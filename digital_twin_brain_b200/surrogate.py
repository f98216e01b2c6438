"""Surrogate forecast of the data-assimilation loop.

:class:`MLP` wraps the ``dtb_mlp_*`` kernels (BF16 weights, FP32 master copy
and accumulation): in -> hidden -> hidden -> 1 with GELU.  :class:`RateSurrogate`
builds its inputs for one (member, region): the 4 g_ui factors and the
region's firing rates of the previous 8 windows, and predicts the next
window's rate (all in log space, standardised).  It is trained on windows the
simulator generates (:func:`collect_windows`).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import DTB_DEVICE, DTB_HOST


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if isinstance(t, torch.Tensor) else t.ctypes.data_as(ctypes.c_void_p)


class MLP:
    def __init__(self, in_dim: int, hidden: int = 256, seed: int = 0, device: int = 0):
        self.in_dim, self.hidden, self.device = in_dim, hidden, device
        self.dev = torch.device("cuda", device)
        h = ctypes.c_void_p()
        _lib.call("dtb_mlp_create", in_dim, hidden, int(seed), device, ctypes.byref(h))
        self._h = h
        n = ctypes.c_int64()
        _lib.call("dtb_mlp_n_params", self._h, ctypes.byref(n))
        self.n_params = int(n.value)
        self._loss = torch.zeros(1, dtype=torch.float32, device=self.dev)

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().dtb_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _stream(self):
        _lib.call("dtb_mlp_set_stream", self._h, ctypes.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream))

    def params(self) -> np.ndarray:
        out = np.empty(self.n_params, np.float32)
        self._stream()
        _lib.call("dtb_mlp_get_params", self._h, _p(out), DTB_HOST)
        return out

    def set_params(self, w: np.ndarray):
        w = np.ascontiguousarray(w, np.float32)
        assert w.size == self.n_params
        self._stream()
        _lib.call("dtb_mlp_set_params", self._h, _p(w), DTB_HOST)

    def forward(self, x: torch.Tensor) -> torch.Tensor:
        x = x.to(self.dev, torch.float32).contiguous()
        y = torch.empty(x.shape[0], dtype=torch.float32, device=self.dev)
        self._stream()
        _lib.call("dtb_mlp_forward", self._h, _p(x), x.shape[0], _p(y))
        return y

    def gradient(self, x: torch.Tensor, t: torch.Tensor):
        x = x.to(self.dev, torch.float32).contiguous()
        t = t.to(self.dev, torch.float32).contiguous()
        g = torch.empty(self.n_params, dtype=torch.float32, device=self.dev)
        self._stream()
        _lib.call("dtb_mlp_gradient", self._h, _p(x), _p(t), x.shape[0], _p(g), _p(self._loss))
        return g, float(self._loss.item())

    def train_step(self, x: torch.Tensor, t: torch.Tensor, lr: float) -> torch.Tensor:
        self._stream()
        _lib.call("dtb_mlp_train_step", self._h, _p(x), _p(t), x.shape[0], float(lr), _p(self._loss))
        return self._loss

    def fit(self, x: torch.Tensor, t: torch.Tensor, epochs: int = 50, batch: int = 4096, lr: float = 1e-3,
            seed: int = 0) -> list:
        """Minibatch Adam; returns the mean training loss of every epoch."""
        x = x.to(self.dev, torch.float32).contiguous()
        t = t.to(self.dev, torch.float32).contiguous()
        g = torch.Generator(device=self.dev)
        g.manual_seed(seed)
        hist = []
        n = x.shape[0]
        for ep in range(epochs):
            perm = torch.randperm(n, generator=g, device=self.dev)
            tot = torch.zeros((), device=self.dev)
            nb = 0
            for i in range(0, n - batch + 1 if n >= batch else 1, batch):
                idx = perm[i:i + batch]
                xb, tb = x[idx].contiguous(), t[idx].contiguous()
                tot += self.train_step(xb, tb, lr)[0]
                nb += 1
            hist.append(float(tot.item()) / max(nb, 1))
        return hist


HISTORY = 8
N_GUI = 4
CONTEXT = 2     # the member's mean rate over all its regions in the last CONTEXT windows


def with_context(hist: torch.Tensor, context: int = CONTEXT) -> torch.Tensor:
    """[M, R, HISTORY] rate histories -> [M * R, HISTORY + context]: every region's own history
    and its member's mean over regions of the last `context` windows (the input the other
    regions send it)."""
    M, R, H = hist.shape
    if context == 0:
        return hist.reshape(-1, H)
    ctx = hist[:, :, H - context:].mean(dim=1, keepdim=True).expand(M, R, context)
    return torch.cat([hist, ctx], dim=2).reshape(-1, H + context)


class RateSurrogate:
    """Next-window firing rate of a region from its g_ui factors, the rates of the previous
    HISTORY windows and its member's mean rate over the last CONTEXT windows (input
    4 + 8 + 2 = 14, hidden 2 x 256 GELU, one output)."""

    def __init__(self, hidden: int = 256, seed: int = 0, device: int = 0, eps: float = 1e-6,
                 context: int = CONTEXT):
        self.context = context
        self.mlp = MLP(N_GUI + HISTORY + context, hidden, seed, device)
        self.dev = self.mlp.dev
        self.eps = eps
        self.mu_x = self.sd_x = None
        self.mu_y = self.sd_y = None

    def features(self, gui: torch.Tensor, hist: torch.Tensor) -> torch.Tensor:
        """gui [n,4] factors, hist [n, HISTORY + context] rates (own history oldest first, then the
        member means) -> standardised log features."""
        x = torch.cat([torch.log(gui.to(self.dev).float()), torch.log(hist.to(self.dev).float() + self.eps)], dim=1)
        if self.mu_x is not None:
            x = (x - self.mu_x) / self.sd_x
        return x

    def fit(self, gui, hist, target, epochs: int = 60, batch: int = 4096, lr: float = 2e-3, seed: int = 0):
        x = torch.cat([torch.log(gui.to(self.dev).float()), torch.log(hist.to(self.dev).float() + self.eps)], dim=1)
        y = torch.log(target.to(self.dev).float() + self.eps)
        self.mu_x, self.sd_x = x.mean(0), x.std(0).clamp_min(1e-6)
        self.mu_y, self.sd_y = y.mean(), y.std().clamp_min(1e-6)
        return self.mlp.fit((x - self.mu_x) / self.sd_x, (y - self.mu_y) / self.sd_y, epochs=epochs, batch=batch,
                            lr=lr, seed=seed)

    def adapt(self, gui, hist, target, steps: int = 20, lr: float = 5e-4):
        """A few Adam steps on new windows, keeping the standardisation of the first fit."""
        x = self.features(gui, hist).contiguous()
        y = ((torch.log(target.to(self.dev).float() + self.eps) - self.mu_y) / self.sd_y).contiguous()
        loss = None
        for _ in range(steps):
            loss = self.mlp.train_step(x, y, lr)
        return float(loss[0].item()) if loss is not None else None

    def predict(self, gui, hist) -> torch.Tensor:
        y = self.mlp.forward(self.features(gui, hist))
        return torch.clamp(torch.exp(y * self.sd_y + self.mu_y) - self.eps, min=0.0)


def _main(argv=None):
    """python -m digital_twin_brain_b200.surrogate [--rows B] [--calls n]: n forward passes and n
    Adam training steps of the surrogate network (14 -> 256 -> 256 -> 1) on B random rows, for
    timing and profiling its tensor-core kernels; prints the mean milliseconds of each."""
    import argparse
    import json
    ap = argparse.ArgumentParser()
    ap.add_argument("--rows", type=int, default=128 * 90)
    ap.add_argument("--calls", type=int, default=5)
    a = ap.parse_args(argv)
    dev = torch.device("cuda", 0)
    m = MLP(N_GUI + HISTORY + CONTEXT, 256, seed=0, device=0)
    g = torch.Generator(device=dev).manual_seed(0)
    x = torch.randn(a.rows, m.in_dim, device=dev, generator=g)
    t = torch.randn(a.rows, device=dev, generator=g)
    out = {}
    for name, fn in (("forward", lambda: m.forward(x)), ("train_step", lambda: m.train_step(x, t, 1e-4))):
        fn()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(a.calls):
            fn()
        e1.record()
        torch.cuda.synchronize(dev)
        out[name + "_ms"] = e0.elapsed_time(e1) / a.calls
    m.close()
    print(json.dumps({"rows": a.rows, **out}))


if __name__ == "__main__":
    _main()
