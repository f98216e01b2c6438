"""Data assimilation on the device: ensemble windows, EnKF analysis, surrogate-served windows."""
import numpy as np
import pytest
import torch

from digital_twin_brain_b200 import synthetic
from digital_twin_brain_b200.assimilation import DAConfig, EnsembleDA, SurrogateDA, collect_windows, log_torch
from digital_twin_brain_b200.surrogate import HISTORY, RateSurrogate

pytestmark = pytest.mark.gpu

TEMPLATE = synthetic.whole_brain(R=6, mean_size=400, sigma=0.3, K=40, gen_seed=3, name="da_small")


def test_ensemble_da_window_and_filter():
    cfg = DAConfig(n_members=12, steps_per_window=400, seed=1)
    da = EnsembleDA(TEMPLATE, cfg)
    da.hp_random_initialize()
    h = da.da_evolve()
    assert h.shape == (12, TEMPLATE.R, 4 + 6) and torch.isfinite(h).all()
    rates = da.window_rates()
    assert rates.shape == (12, TEMPLATE.R) and (rates > 0).all()
    obs = h[:, :, -1].mean(0)
    before = da.hp_log.clone()
    da.da_filter(obs)
    assert not torch.equal(before, da.hp_log)
    np.testing.assert_allclose(da.net.get_bold("s")[da.region_idx.reshape(-1)],
                               da.hidden[:, :, -5].reshape(-1).double().cpu().numpy(), rtol=1e-6)


def test_member_hp_changes_its_own_rate():
    cfg = DAConfig(n_members=2, steps_per_window=1500, seed=2)
    da = EnsembleDA(TEMPLATE, cfg)
    hp = torch.ones(2, TEMPLATE.R * 4, device=da.dev)
    hp[1, 0::4] = 1.45      # more AMPA in member 1
    hp[1, 2::4] = 0.55      # less GABAa
    da.hp_log = log_torch(hp.clamp(0.51, 1.49), da.low, da.high)
    da.apply_hp()
    da.evolve()
    r = da.window_rates()
    assert (r[1] > r[0]).mean() >= 0.8


def test_surrogate_da_runs_with_judges_and_fallback():
    cfg = DAConfig(n_members=12, steps_per_window=300, seed=3)
    g, h, t = collect_windows(TEMPLATE, cfg, windows=10)
    assert g.shape[0] == h.shape[0] == t.shape[0] == 2 * 12 * TEMPLATE.R and h.shape[1] == 8 + 2
    sur = RateSurrogate(seed=0)
    sur.fit(g, h, t, epochs=5)
    sda = SurrogateDA(TEMPLATE, cfg, sur, n_judge=4, threshold=0.0)     # always falls back
    obs = torch.full((3, TEMPLATE.R), 0.02, device=sda.dev)
    res = sda.run(obs)
    assert res["fallbacks"] == 3 and np.isfinite(res["bold_pred"]).all()
    sda2 = SurrogateDA(TEMPLATE, cfg, sur, n_judge=4, threshold=1e9)    # never falls back
    res2 = sda2.run(obs)
    assert res2["fallbacks"] == 0 and np.isfinite(res2["bold_pred"]).all()
    # adaptation, residual spread and judge-based BOLD correction on served windows
    sda3 = SurrogateDA(TEMPLATE, cfg, sur, n_judge=4, threshold=1e9, adapt_steps=3, spread=True, bias_correct=True)
    sda3.hp_random_initialize()
    sda3.burn_in(2)
    res3 = sda3.run(obs)
    assert res3["fallbacks"] == 0 and np.isfinite(res3["bold_pred"]).all()
    # the forecast of a window from the surrogate adapted on half of that window's judges; the
    # other members' start histories forecast from their own g_ui, every BOLD state restarted
    sda4 = SurrogateDA(TEMPLATE, cfg, sur, n_judge=4, threshold=1e9, adapt_steps=3, adapt_split=True,
                       self_history=True)
    sda4.hp_random_initialize()
    sda4.burn_in(1)
    assert not torch.equal(sda4.hist[4], sda4.hist[5])          # members' own histories
    jb = sda4.judge.get_bold_state()
    assert torch.all(jb[..., 0] == 0) and torch.all(jb[..., 2] == 1) and torch.all(jb[..., 3] == 1)
    res4 = sda4.run(obs)
    assert res4["fallbacks"] == 0 and np.isfinite(res4["bold_pred"]).all() and len(res4["errors"]) == 3


def test_surrogate_adapt_lowers_loss_on_new_windows():
    torch.manual_seed(0)
    g = torch.rand(2000, 4) + 0.5
    h = torch.rand(2000, 10) * 0.01 + 1e-3
    t = h.mean(1) * g[:, 0]
    sur = RateSurrogate(seed=1)
    sur.fit(g[:1000], h[:1000], t[:1000] * 0.5, epochs=5)     # trained on a shifted relation
    before = sur.adapt(g[1000:], h[1000:], t[1000:], steps=1)
    after = sur.adapt(g[1000:], h[1000:], t[1000:], steps=40)
    assert after < before


def test_surrogate_beats_persistence_on_simulated_windows():
    """Trained on windows this simulator generates, the surrogate forecasts held-out windows'
    rates better than the method without it (the previous window's rate)."""
    template = synthetic.whole_brain(R=8, mean_size=1500, sigma=0.3, K=60, gen_seed=5, name="da_sur",
                                     g_ui=tuple(x * y for x, y in zip(synthetic.LIF["g_ui"], (2.0, 2.0, 1.0, 1.0))))
    cfg = DAConfig(n_members=32, steps_per_window=1500, seed=4, hp_sigma=1.0)
    g, h, t = collect_windows(template, cfg, windows=20)
    n = g.shape[0]
    perm = torch.from_numpy(np.random.default_rng(0).permutation(n))
    tr, te = perm[: int(0.85 * n)], perm[int(0.85 * n):]
    sur = RateSurrogate(seed=3)
    sur.fit(g[tr], h[tr], t[tr], epochs=60)
    eps = 1e-6
    pred = sur.predict(g[te], h[te]).cpu()
    err_net = float(torch.sqrt(torch.mean((torch.log(pred + eps) - torch.log(t[te] + eps)) ** 2)))
    err_persist = float(torch.sqrt(torch.mean((torch.log(h[te][:, HISTORY - 1] + eps) - torch.log(t[te] + eps)) ** 2)))
    assert err_net < 0.9 * err_persist, (err_net, err_persist)
