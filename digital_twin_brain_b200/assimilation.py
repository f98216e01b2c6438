"""Data assimilation on one GPU: the ensemble Kalman filter loop of
``data_assimilation/DataAssimilation.py`` over a batched ensemble network.

* :func:`diffusion_enkf` — ``DataAssimilation.py:40-60`` (same operation
  order, torch on the ensemble's device);
* :func:`log_torch`, :func:`sigmoid_torch` — the bounded hyper-parameter
  transform (``DataAssimilation.py:111-140``);
* :class:`EnsembleDA` — ``hp_random_initialize`` (``:204-252``), ``da_evolve``
  (``:353-370``), ``da_filter`` (``:372-400``) and ``da_rest_run``
  (``:402-453``) with all members stepped together on the device: members
  are copies of one template network (same connectivity, own noise streams),
  each region's g_ui scaled by its member's hyper-parameters
  (``mul_property_by_subblk``, ``dist_blockwrapper_pytorch.py:446``), BOLD
  per (member, region) fused into the step (``simulation.py:269-279``).

The hidden state of a (member, region) is [hp_log (n_hp), act, s, q, v, f_in,
bold] as ``DataAssimilation.get_hidden_state`` builds it (``:327-351``).
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import synthetic
from .network import Network
from .surrogate import with_context


def diffusion_enkf(w_hat: torch.Tensor, bold_sigma: float, bold_t: torch.Tensor, solo_rate: float,
                   noise: torch.Tensor | None = None, generator: torch.Generator | None = None) -> torch.Tensor:
    """DataAssimilation.py:40-60.  w_hat [E, R, S] (last column = BOLD), bold_t [1, R].
    noise: standard-normal [E, R] observation perturbations (drawn when None)."""
    ensembles, brain_num, state_num = w_hat.shape
    w = w_hat.clone()
    w_mean = torch.mean(w_hat, dim=0, keepdim=True)
    w_diff = w_hat - w_mean
    w_cx = w_diff[:, :, -1] * w_diff[:, :, -1]
    w_cxx = torch.sum(w_cx, dim=0) / (ensembles - 1) + bold_sigma
    temp = w_diff[:, :, -1] / (w_cxx.reshape([1, brain_num])) / (ensembles - 1)
    if noise is None:
        noise = torch.normal(0, 1, size=(ensembles, brain_num), generator=generator, device=w_hat.device)
    bold_with_noise = bold_t + bold_sigma ** 0.5 * noise.type_as(bold_t)
    w += solo_rate * (bold_with_noise - w_hat[:, :, -1])[:, :, None] * torch.sum(temp[:, :, None] * w_diff, dim=0,
                                                                                 keepdim=True)
    w += (1 - solo_rate) * torch.mm(torch.mm(bold_with_noise - w_hat[:, :, -1], temp.T) / brain_num,
                                    w_diff.reshape([ensembles, -1])).reshape(w_hat.shape)
    return w


def log_torch(val, lower, upper, scale=10):
    """DataAssimilation.py:111-125 (inverse of sigmoid_torch)."""
    shape = val.shape
    val = val.reshape(-1, lower.shape[-1])
    return (scale * (torch.log(val - lower) - torch.log(upper - val))).reshape(shape)


def sigmoid_torch(val, lower, upper, scale=10):
    """DataAssimilation.py:128-140: lower + (upper - lower) * sigmoid(val / scale)."""
    shape = val.shape
    val = val.reshape(-1, lower.shape[-1])
    return (lower + (upper - lower) * torch.sigmoid(val / scale)).reshape(shape)


@dataclass
class DAConfig:
    n_members: int = 128
    steps_per_window: int = 8000          # 800 ms at dt = 0.1 ms
    hp_cols: tuple = (10, 11, 12, 13)      # g_ui property columns assimilated (AMPA, NMDA, GABAa, GABAb)
    hp_low: float = 0.5                   # bounds as factors of the template g_ui
    hp_high: float = 1.5
    hp_sigma: float = 0.25                # random-walk variance (DataAssimilation.da_evolve default)
    bold_sigma: float = 1e-8
    solo_rate: float = 0.8
    bound: float | None = 40.0
    noise_rate: float | None = None       # None: per-neuron property column 0
    seed: int = 0
    extra: dict = field(default_factory=dict)


class EnsembleDA:
    """DataAssimilation restated over one batched ensemble network on one GPU."""

    def __init__(self, template: synthetic.NetworkSpec, cfg: DAConfig, device: int = 0, members=None):
        self.cfg = cfg
        self.template = template
        self.device = device
        self.dev = torch.device("cuda", device)
        M = cfg.n_members if members is None else len(members)
        self.M = M
        self.R = template.R
        self.n_hp = len(cfg.hp_cols)
        self.spec = synthetic.ensemble([template] * M, name=f"da_{M}x{template.R}")
        self.net = Network.from_spec(self.spec, device=device)
        self.net.attach_bold(self.spec.sub_to_region(), self.spec.R, delta_t=template.dt / 1000.0)
        # global region of (member, region)
        self.region_idx = np.array([[synthetic.member_region_index(self.spec, m, r) for r in range(self.R)]
                                    for m in range(M)], np.int64)
        self.low = torch.full((self.R * self.n_hp,), cfg.hp_low, dtype=torch.float32, device=self.dev)
        self.high = torch.full((self.R * self.n_hp,), cfg.hp_high, dtype=torch.float32, device=self.dev)
        self.gen = torch.Generator(device=self.dev)
        self.gen.manual_seed(cfg.seed)
        self.rng = np.random.default_rng(cfg.seed)
        self.hp_log = None
        self.hidden = None
        self.steps = 0

    # ------------------------------------------------------------ parameters
    def hp_random_initialize(self):
        """DataAssimilation.py:204-252 (method 1: linspace in logit space, shuffled per parameter)."""
        temp = torch.linspace(-1 / 3, 1 / 3, self.M)
        hp_log = 10 * (torch.log(temp + 1) - torch.log(1 - temp)).repeat_interleave(self.R * self.n_hp)
        hp_log = hp_log.reshape(self.M, self.R, self.n_hp)
        for i in range(self.n_hp):
            idx = torch.from_numpy(self.rng.permutation(self.M))
            hp_log[:, :, i] = hp_log[idx, :, i]
        self.hp_log = hp_log.reshape(self.M, -1).to(self.dev)
        self.apply_hp()
        return self.hp

    @property
    def hp(self) -> torch.Tensor:
        return sigmoid_torch(self.hp_log, self.low, self.high)

    def apply_hp(self, hp: torch.Tensor | None = None):
        """mul_property_by_subblk: g_ui column c of both populations of (member, region) = base * hp."""
        hp = (self.hp if hp is None else hp).reshape(self.M, self.R, self.n_hp).detach().cpu().numpy()
        reg = self.region_idx                                   # [M, R]
        subs = np.stack([2 * reg, 2 * reg + 1], axis=-1)        # [M, R, 2]
        sub = np.broadcast_to(subs[:, :, None, :], (self.M, self.R, self.n_hp, 2))
        col = np.broadcast_to(np.asarray(self.cfg.hp_cols, np.int32)[None, None, :, None], sub.shape)
        val = np.broadcast_to(hp[:, :, :, None], sub.shape)
        self.net.scale_property_by_subblock(sub.reshape(-1), col.reshape(-1), val.reshape(-1))

    # ------------------------------------------------------------ evolution
    def evolve(self, steps: int | None = None) -> torch.Tensor:
        """Run one window and return [M, R, 6]: act, s, q, v, f_in, bold (simulation.evolve bold_detail)."""
        steps = self.cfg.steps_per_window if steps is None else steps
        self.net.clear_window_spikes()
        self.net.run(steps, noise_rate=self.cfg.noise_rate, mode="push", out=None)
        self.steps += steps
        idx = torch.from_numpy(self.region_idx.reshape(-1)).to(self.dev)
        cols = [self.net.get_bold(f, device=True)[idx] for f in ("act", "s", "q", "v", "f_in", "bold")]
        return torch.stack(cols, dim=-1).reshape(self.M, self.R, 6).float()

    def window_rates(self) -> np.ndarray:
        """Mean spikes per neuron per step of every (member, region) over the last window."""
        spk = self.net.window_spikes().astype(np.float64)
        cnt = self.net.get(9).astype(np.float64)              # FIELD_SUB_COUNT
        reg = self.region_idx
        s = spk[2 * reg] + spk[2 * reg + 1]
        n = cnt[2 * reg] + cnt[2 * reg + 1]
        return s / np.maximum(n, 1.0) / max(self.cfg.steps_per_window, 1)

    def hidden_state(self, out6: torch.Tensor) -> torch.Tensor:
        return torch.cat([self.hp_log.reshape(self.M, self.R, self.n_hp), out6], dim=2)

    def da_evolve(self) -> torch.Tensor:
        """DataAssimilation.py:353-370."""
        self.hp_log = self.hp_log + math.sqrt(self.cfg.hp_sigma) * torch.randn(self.hp_log.shape, generator=self.gen,
                                                                               device=self.dev)
        self.apply_hp()
        self.hidden = self.hidden_state(self.evolve())
        return self.hidden

    def get_bold_state(self) -> torch.Tensor:
        """The (member, region) BOLD states s, q, v, f_in as [M, R, 4] (float64, device)."""
        idx = self.region_idx.reshape(-1)
        cols = [torch.from_numpy(self.net.get_bold(f)[idx]) for f in ("s", "q", "v", "f_in")]
        return torch.stack(cols, dim=-1).reshape(self.M, self.R, 4).to(self.dev)

    def reset_bold_state(self):
        """The (member, region) BOLD states back to their initial values s = q = 0, v = f_in = 1."""
        idx = self.region_idx.reshape(-1)
        for f, v0 in (("s", 0.0), ("q", 0.0), ("v", 1.0), ("f_in", 1.0)):
            full = self.net.get_bold(f)
            full[idx] = v0
            self.net.set_bold(f, full)

    def set_bold_state(self, sqvf: torch.Tensor):
        """bold.state_update (bold_model_pytorch.py:34-41) for the (member, region) BOLD states."""
        idx = self.region_idx.reshape(-1)
        for k, f in enumerate(("s", "q", "v", "f_in")):
            full = self.net.get_bold(f)
            v = sqvf[:, :, k].reshape(-1).double().cpu().numpy()
            if k > 0:
                v = np.where(np.isnan(v), v, np.maximum(v, 1e-5))
            full[idx] = v
            self.net.set_bold(f, full)

    def da_filter(self, bold_obs: torch.Tensor, noise: torch.Tensor | None = None) -> torch.Tensor:
        """DataAssimilation.py:372-400."""
        self.hidden = diffusion_enkf(self.hidden, self.cfg.bold_sigma, bold_obs.reshape(1, -1).to(self.hidden),
                                     self.cfg.solo_rate, noise=noise, generator=self.gen)
        self.hp_log = self.hidden[:, :, :self.n_hp].reshape(self.M, -1).clone()
        if self.cfg.bound is not None:
            self.hp_log = torch.clamp(self.hp_log, -self.cfg.bound, self.cfg.bound)
        self.set_bold_state(self.hidden[:, :, -5:-1])
        return self.hidden

    def run(self, bold_obs: torch.Tensor, windows: int | None = None, warmup_steps: int = 0) -> dict:
        """DataAssimilation.da_rest_run (:402-453) without the file output: returns the per-window
        predicted BOLD (before filtering), hp means and timings."""
        T = bold_obs.shape[0] if windows is None else windows
        if self.hp_log is None:
            self.hp_random_initialize()
        if warmup_steps:
            self.net.run(warmup_steps, noise_rate=self.cfg.noise_rate, mode="push", out=None)
        bold_pred, hp_mean, times = [], [], []
        for t in range(T):
            torch.cuda.synchronize(self.dev)
            t0 = time.perf_counter()
            h = self.da_evolve()
            bold_pred.append(h[:, :, -1].mean(0).cpu().numpy())
            self.da_filter(bold_obs[t].to(self.dev))
            hp_mean.append(self.hp.reshape(self.M, self.R, self.n_hp).mean(0).cpu().numpy())
            torch.cuda.synchronize(self.dev)
            times.append(time.perf_counter() - t0)
        return dict(bold_pred=np.stack(bold_pred), hp_mean=np.stack(hp_mean), window_s=np.array(times))


def judge_error(pred: torch.Tensor, rates: torch.Tensor) -> float:
    """The judges' score: absolute error of the window rates relative to their total, so that
    quiet regions (whose BOLD barely depends on their rate) do not dominate."""
    return (torch.sum(torch.abs(pred - rates)) / (torch.sum(rates) + 1e-5 * rates.numel())).item()


class SurrogateDA:
    """EnKF data assimilation whose forecast comes from the surrogate for most members.

    Members 0..n_judge-1 run the simulator every window (the judges); the
    surrogate predicts every member's window rate from its g_ui factors and
    rate history, the surrogate members' hemodynamics are integrated from
    that rate (dtb_bold_run_steps), and the judges score the surrogate on
    their simulated rates: when their error (``judge_error``) exceeds `threshold`
    (calibrate it on held-out windows: a margin over the surrogate's validated error),
    the window is recomputed for the surrogate members on the simulator
    (fallback).  The analysis step is the same diffusion EnKF over all members.

    adapt_split: the judges' window also serves the forecast of the same window:
    the surrogate first adapts on the first half of the judges, then forecasts every
    member, is scored on the other half (windows it has not seen) and finally adapts
    on that half too.  Without it the forecast comes from the surrogate as adapted up
    to the previous window and every judge scores it.

    self_history: after the burn-in, the members off the simulator start from rate
    histories the surrogate forecasts from their own g_ui (iterated on its own output)
    instead of the judges' regional mean, and the judges' BOLD state restarts from the
    initial state, so that every member's hemodynamics start together at the first window.
    """

    def __init__(self, template: synthetic.NetworkSpec, cfg: DAConfig, surrogate, n_judge: int = 16,
                 threshold: float = 0.3, device: int = 0, adapt_steps: int = 0, adapt_lr: float = 5e-4,
                 bias_correct: bool = False, spread: bool = False, adapt_split: bool = False,
                 self_history: bool = False):
        from .network import BoldModel
        from .surrogate import HISTORY
        self.cfg = cfg
        self.M = cfg.n_members
        self.J = n_judge
        self.R = template.R
        self.n_hp = len(cfg.hp_cols)
        self.dev = torch.device("cuda", device)
        self.device = device
        self.template = template
        self.sur = surrogate
        self.threshold = threshold
        self.adapt_steps = adapt_steps
        self.adapt_lr = adapt_lr
        self.adapt_split = adapt_split and adapt_steps > 0 and n_judge >= 2
        self.self_history = self_history
        jcfg = DAConfig(**{**cfg.__dict__, "n_members": n_judge})
        self.judge = EnsembleDA(template, jcfg, device)
        self.full = None   # fallback simulator for the surrogate members (built on first use)
        self.bold = BoldModel(n_regions=(self.M - self.J) * self.R, dtype=torch.float64, delta_t=template.dt / 1000.0,
                              device=device)
        # bias_correct: the judges' BOLD is also integrated from their surrogate rates; the mean
        # difference to their simulated BOLD (per region) corrects the surrogate members' BOLD
        self.bias_correct = bias_correct
        # spread: surrogate rates get the judges' log-residual spread (mean-preserving lognormal
        # noise), so the forecast ensemble keeps the variability simulated members have
        self.spread = spread
        self.jbold = BoldModel(n_regions=self.J * self.R, dtype=torch.float64, delta_t=template.dt / 1000.0,
                               device=device) if bias_correct else None
        self.low = self.judge.low
        self.high = self.judge.high
        self.gen = torch.Generator(device=self.dev)
        self.gen.manual_seed(cfg.seed)          # the same random walk and perturbations as EnsembleDA
        self.rng = np.random.default_rng(cfg.seed)
        self.hist = None   # [M, R, HISTORY] window rates
        self.H = HISTORY
        self.hp_log = None
        self.hidden = None
        self.fallbacks = 0
        self.errors = []

    def hp_random_initialize(self):
        temp = torch.linspace(-1 / 3, 1 / 3, self.M)
        hp_log = 10 * (torch.log(temp + 1) - torch.log(1 - temp)).repeat_interleave(self.R * self.n_hp)
        hp_log = hp_log.reshape(self.M, self.R, self.n_hp)
        for i in range(self.n_hp):
            idx = torch.from_numpy(self.rng.permutation(self.M))
            hp_log[:, :, i] = hp_log[idx, :, i]
        self.hp_log = hp_log.reshape(self.M, -1).to(self.dev)

    @property
    def hp(self):
        return sigmoid_torch(self.hp_log, self.low, self.high)

    def burn_in(self, windows: int = 1, steps: int | None = None):
        """`windows` judge windows before the assimilation seed the rate histories: the judges'
        own, and the judges' regional mean for every other member.  With adaptation on, the
        surrogate also learns from each of these windows."""
        self.judge.hp_log = self.hp_log[:self.J].clone()
        self.judge.apply_hp()
        gui = self.hp.reshape(self.M, self.R, self.n_hp)[:self.J].reshape(-1, self.n_hp)
        jh = None
        for _ in range(max(1, windows)):
            self.judge.evolve(steps)
            r = torch.from_numpy(self.judge.window_rates()).to(self.dev).float()      # [J, R]
            if jh is not None and self.adapt_steps:
                h = torch.cat([jh[:, :, :1].repeat(1, 1, self.H - jh.shape[2]), jh], 2) if jh.shape[2] < self.H else jh
                self.sur.adapt(gui, with_context(h, self.sur.context), r.reshape(-1), steps=self.adapt_steps,
                               lr=self.adapt_lr)
            jh = r[:, :, None] if jh is None else torch.cat([jh, r[:, :, None]], 2)[:, :, -self.H:]
        if jh.shape[2] < self.H:
            jh = torch.cat([jh[:, :, :1].repeat(1, 1, self.H - jh.shape[2]), jh], 2)
        self.hist = jh.mean(0, keepdim=True).repeat(self.M, 1, 1)
        self.hist[:self.J] = jh
        if self.self_history and self.M > self.J:
            # the other members' histories from their own g_ui: the surrogate iterated on its own
            # forecasts, HISTORY times, starting from the judges' regional mean
            g_s = self.hp.reshape(self.M, self.R, self.n_hp)[self.J:].reshape(-1, self.n_hp)
            for _ in range(self.H):
                p = self.sur.predict(g_s, with_context(self.hist[self.J:], self.sur.context)).reshape(self.M - self.J,
                                                                                                    self.R)
                self.hist[self.J:] = torch.cat([self.hist[self.J:, :, 1:], p[:, :, None]], dim=2)
            # every member's hemodynamics from the initial state at the first window, as in an
            # all-simulator run (the judges' burn-in windows only warm their neurons)
            self.judge.reset_bold_state()

    def _fallback(self, hp_s: torch.Tensor, bold_sqvf: torch.Tensor):
        if self.full is None:
            fcfg = DAConfig(**{**self.cfg.__dict__, "n_members": self.M - self.J})
            self.full = EnsembleDA(self.template, fcfg, self.device)
        self.full.hp_log = log_torch(hp_s.reshape(self.M - self.J, -1), self.low, self.high)
        self.full.apply_hp()
        self.full.set_bold_state(bold_sqvf)
        out6 = self.full.evolve()
        rates = torch.from_numpy(self.full.window_rates()).to(self.dev).float()
        return out6, rates

    def da_window(self, bold_obs: torch.Tensor):
        cfg = self.cfg
        self.hp_log = self.hp_log + math.sqrt(cfg.hp_sigma) * torch.randn(self.hp_log.shape, generator=self.gen,
                                                                          device=self.dev)
        hp = self.hp.reshape(self.M, self.R, self.n_hp)
        # judges: simulator
        self.judge.hp_log = self.hp_log[:self.J].clone()
        self.judge.apply_hp()
        jstate = self.judge.get_bold_state() if self.bias_correct else None
        out_j = self.judge.evolve()
        rates_j = torch.from_numpy(self.judge.window_rates()).to(self.dev).float()
        # surrogate forecast of every member's window rate
        gui = hp.reshape(-1, self.n_hp)
        ctx = with_context(self.hist, self.sur.context)
        Ja = self.J // 2 if self.adapt_split else 0      # judges the surrogate adapts on before forecasting
        if Ja:
            self.sur.adapt(gui[:Ja * self.R], ctx[:Ja * self.R], rates_j[:Ja].reshape(-1), steps=self.adapt_steps,
                           lr=self.adapt_lr)
        pred = self.sur.predict(gui, ctx).reshape(self.M, self.R)
        # judge score on the judges the surrogate has not seen this window: symmetric relative
        # error of the window rates (floor 1e-5 spikes/step ~ 0.1 Hz)
        err = judge_error(pred[Ja:self.J], rates_j[Ja:])
        self.errors.append(err)
        if self.adapt_steps:   # the judges' fresh windows refine the surrogate (scored before it learns them)
            self.sur.adapt(gui[Ja * self.R:self.J * self.R], ctx[Ja * self.R:self.J * self.R], rates_j[Ja:].reshape(-1),
                           steps=self.adapt_steps, lr=self.adapt_lr)
        sqvf = torch.stack([self.bold.get(k) for k in range(4)], dim=-1).reshape(self.M - self.J, self.R, 4)
        if err > self.threshold:
            self.fallbacks += 1
            out_s, rates_s = self._fallback(hp[self.J:], sqvf)
            self.bold.set(0, out_s[:, :, 1].double()); self.bold.set(1, out_s[:, :, 2].double())
            self.bold.set(2, out_s[:, :, 3].double()); self.bold.set(3, out_s[:, :, 4].double())
        else:
            rates_s = pred[self.J:]
            if self.spread:
                eps = 1e-6
                res = torch.log(rates_j[Ja:] + eps) - torch.log(pred[Ja:self.J] + eps)
                sd = float(res.std())
                z = torch.randn(rates_s.shape, generator=self.gen, device=self.dev)
                rates_s = rates_s * torch.exp(sd * z - 0.5 * sd * sd)
            sig = self.bold.run_steps(rates_s.reshape(-1).double(), cfg.steps_per_window, 1e-5)
            if self.bias_correct:
                for k in range(4):
                    v = jstate[:, :, k].reshape(-1)
                    self.jbold.set(k, v if k == 0 else torch.clamp(v, min=1e-5))
                sig_j = self.jbold.run_steps(pred[:self.J].reshape(-1).double(), cfg.steps_per_window, 1e-5)
                bias = (out_j[:, :, 5].double() - sig_j.reshape(self.J, self.R)).mean(0)      # [R]
                sig = (sig.reshape(self.M - self.J, self.R) + bias).reshape(-1)
            st = [self.bold.get(k).float() for k in range(4)]
            out_s = torch.stack([rates_s.reshape(-1)] + st + [sig.float()], dim=-1).reshape(self.M - self.J, self.R, 6)
        out6 = torch.cat([out_j, out_s], dim=0)
        rates = torch.cat([rates_j, rates_s], dim=0)
        self.hist = torch.cat([self.hist[:, :, 1:], rates[:, :, None]], dim=2)
        self.hidden = torch.cat([self.hp_log.reshape(self.M, self.R, self.n_hp), out6], dim=2)
        pred_bold = self.hidden[:, :, -1].mean(0)
        # analysis
        self.hidden = diffusion_enkf(self.hidden, cfg.bold_sigma, bold_obs.reshape(1, -1).to(self.hidden),
                                     cfg.solo_rate, generator=self.gen)
        self.hp_log = self.hidden[:, :, :self.n_hp].reshape(self.M, -1).clone()
        if cfg.bound is not None:
            self.hp_log = torch.clamp(self.hp_log, -cfg.bound, cfg.bound)
        st = self.hidden[:, :, -5:-1]
        self.judge.set_bold_state(st[:self.J])
        for k in range(4):
            v = st[self.J:, :, k].reshape(-1).double()
            self.bold.set(k, v if k == 0 else torch.clamp(v, min=1e-5))
        return pred_bold

    def run(self, bold_obs: torch.Tensor, windows: int | None = None) -> dict:
        T = bold_obs.shape[0] if windows is None else windows
        if self.hp_log is None:
            self.hp_random_initialize()
        if self.hist is None:
            self.burn_in()
        bold_pred, hp_mean, times = [], [], []
        for t in range(T):
            torch.cuda.synchronize(self.dev)
            t0 = time.perf_counter()
            pb = self.da_window(bold_obs[t].to(self.dev))
            bold_pred.append(pb.cpu().numpy())
            hp_mean.append(self.hp.reshape(self.M, self.R, self.n_hp).mean(0).cpu().numpy())
            torch.cuda.synchronize(self.dev)
            times.append(time.perf_counter() - t0)
        return dict(bold_pred=np.stack(bold_pred), hp_mean=np.stack(hp_mean), window_s=np.array(times),
                    fallbacks=self.fallbacks, errors=np.array(self.errors))


def collect_da_windows(template: synthetic.NetworkSpec, cfg: DAConfig, bold_obs: torch.Tensor, device: int = 0,
                       history: int = 8, context: int | None = None):
    """Training windows for the surrogate from an assimilation run (every member on the
    simulator, data_assimilation/DataAssimilation.py:402-453) against observations of another
    hidden truth: the g_ui factors of every window then move as the analysis moves them (large
    steps in the first windows), which a random walk does not show.  Returns what
    collect_windows returns, over the windows with a full history."""
    from .surrogate import CONTEXT
    context = CONTEXT if context is None else context
    da = EnsembleDA(template, cfg, device)
    da.hp_random_initialize()
    hps, rates = [], []
    for t in range(bold_obs.shape[0]):
        da.da_evolve()
        hps.append(da.hp.reshape(da.M, da.R, da.n_hp).cpu())
        rates.append(torch.from_numpy(da.window_rates()).float())
        da.da_filter(bold_obs[t].to(da.dev))
    hp = torch.stack(hps)
    rt = torch.stack(rates)
    g, h, t = [], [], []
    for w in range(history, len(hps)):
        g.append(hp[w].reshape(-1, 4))
        h.append(with_context(rt[w - history:w].permute(1, 2, 0), context))
        t.append(rt[w].reshape(-1))
    # the first windows (short histories padded with their earliest rate), where the analysis
    # moves the parameters most
    for w in range(1, min(history, len(hps))):
        hw = rt[:w].permute(1, 2, 0)
        hw = torch.cat([hw[:, :, :1].repeat(1, 1, history - w), hw], 2)
        g.append(hp[w].reshape(-1, 4))
        h.append(with_context(hw, context))
        t.append(rt[w].reshape(-1))
    del da
    return torch.cat(g), torch.cat(h), torch.cat(t)


def collect_windows(template: synthetic.NetworkSpec, cfg: DAConfig, windows: int, device: int = 0,
                    history: int = 8, context: int | None = None):
    """Training windows for the surrogate: an ensemble with random-walk g_ui factors (the DA
    forecast without analysis); returns (gui [n,4], hist [n, history + context], target [n])
    over all (member, region, window) with a full history (see surrogate.with_context)."""
    from .surrogate import CONTEXT
    context = CONTEXT if context is None else context
    da = EnsembleDA(template, cfg, device)
    da.hp_random_initialize()
    hps, rates = [], []
    for w in range(windows):
        da.hp_log = da.hp_log + math.sqrt(cfg.hp_sigma) * torch.randn(da.hp_log.shape, generator=da.gen,
                                                                      device=da.dev)
        da.apply_hp()
        da.evolve()
        hps.append(da.hp.reshape(da.M, da.R, da.n_hp).cpu())
        rates.append(torch.from_numpy(da.window_rates()).float())
    hp = torch.stack(hps)            # [W, M, R, 4]
    rt = torch.stack(rates)          # [W, M, R]
    g, h, t = [], [], []
    for w in range(history, windows):
        g.append(hp[w].reshape(-1, 4))
        h.append(with_context(rt[w - history:w].permute(1, 2, 0), context))
        t.append(rt[w].reshape(-1))
    del da
    return torch.cat(g), torch.cat(h), torch.cat(t)
