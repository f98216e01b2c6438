"""Data-assimilation window benchmark: surrogate-served vs all-simulator ensemble.

    python -m digital_twin_brain_b200.da_bench [--members 128] [--judges 8] [--regions 90]
        [--region-size 2000] [--windows 50] [--steps-per-window 8000] [--train-windows 18] [--out FILE]

1. Truth: one network with hidden true g_ui factors (per region, 4 receptors)
   runs `windows` windows; its BOLD at the end of every window plus Gaussian
   noise (sigma = 0.1 x the per-region std over windows) is the observation.
2. Plain: EnsembleDA with every member on the simulator
   (data_assimilation/DataAssimilation.py:402-453 restated).
3. Surrogate: training windows from an assimilation run against another
   hidden truth and from a random-walk ensemble, RateSurrogate trained on
   them, then SurrogateDA: judges on the simulator, the rest forecast by the
   network, which adapts on half of each window's judges before forecasting
   that window and is scored on the other half (fallback on judge error); the
   members off the simulator start from histories forecast from their own g_ui.
Reports mean window time of both, their ratio, the BOLD-fit RMSE of the
ensemble-mean forecast against the observation, and the g_ui recovery error.
The reference's 2e5 neurons per region do not fit 128 members on one GPU
(~3 TB of synapses); --region-size scales every region (stated in the output).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from . import synthetic
from .assimilation import (DAConfig, EnsembleDA, SurrogateDA, collect_da_windows, collect_windows, judge_error,
                           log_torch)
from .surrogate import HISTORY, RateSurrogate


def observe(template, hp_true: torch.Tensor, windows: int, base: dict, seed: int) -> torch.Tensor:
    """BOLD at the end of every window of one network with the hidden g_ui factors hp_true
    [R, 4], plus Gaussian noise of 0.1 x the per-region std over the windows: [windows, R]."""
    dev = hp_true.device
    truth = EnsembleDA(template, DAConfig(n_members=1, **base))
    truth.hp_log = log_torch(hp_true.reshape(1, -1), truth.low, truth.high)
    truth.apply_hp()
    bold_true = torch.stack([truth.evolve()[0, :, -1].double() for _ in range(windows)])   # [W, R]
    del truth
    sd = bold_true.std(0, keepdim=True).clamp_min(1e-9)
    noise = torch.randn(bold_true.shape, device=dev, dtype=torch.float64,
                        generator=torch.Generator(device=dev).manual_seed(seed))
    return (bold_true + 0.1 * sd * noise).float()


def main(argv=None, quiet: bool = False) -> dict:
    """Runs the comparison with command-line style arguments; returns the result dict
    (and prints it as one JSON line unless quiet)."""
    ap = argparse.ArgumentParser()
    ap.add_argument("--members", type=int, default=128)
    ap.add_argument("--judges", type=int, default=8)
    ap.add_argument("--regions", type=int, default=90)
    ap.add_argument("--region-size", type=float, default=2000)
    ap.add_argument("--K", type=int, default=100)
    ap.add_argument("--windows", type=int, default=50)
    ap.add_argument("--steps-per-window", type=int, default=8000)
    ap.add_argument("--train-windows", type=int, default=30)
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--train-sigma", type=float, default=2.0,
                    help="random-walk variance of the training ensemble (wider than the DA walk for coverage)")
    ap.add_argument("--train-source", default="both", choices=["da", "walk", "both"],
                    help="da: training windows from an assimilation run against another hidden truth (its "
                         "analysis steps move the parameters as the served run's do); walk: a random-walk "
                         "ensemble; both: the two sets together")
    ap.add_argument("--threshold", type=float, default=None,
                    help="judge fallback threshold (default: --margin x the held-out judge error of the surrogate)")
    ap.add_argument("--margin", type=float, default=2.0)
    ap.add_argument("--burn-in-windows", type=int, default=1,
                    help="judge windows before the assimilation (histories, surrogate adaptation); timed")
    ap.add_argument("--spread", type=int, default=0,
                    help="give the surrogate members' rates the judges' residual spread")
    ap.add_argument("--bias-correct", type=int, default=0,
                    help="correct the surrogate members' BOLD by the judges' simulated-minus-surrogate mean")
    ap.add_argument("--self-history", type=int, default=1,
                    help="1: members off the simulator start from surrogate-forecast histories of their own g_ui, "
                         "and every member's BOLD starts at the first window")
    ap.add_argument("--adapt-split", type=int, default=1,
                    help="1: adapt on half of each window's judges before forecasting that window, score on the other half")
    ap.add_argument("--adapt-steps", type=int, default=60,
                    help="Adam steps per window on the judges' windows (0: the surrogate stays as trained)")
    ap.add_argument("--gain", type=float, default=2.0,
                    help="excitatory g_ui of the template as a multiple of the single-block values (2.0: ~6 Hz)")
    ap.add_argument("--skip", type=int, default=5, help="windows excluded from the RMSE (spin-up)")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--plain-seeds", type=int, default=2,
                    help="plain runs with different DA seeds (their RMSE spread is the yardstick for the surrogate)")
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    dev = torch.device("cuda", 0)
    t_all = time.perf_counter()
    g0 = synthetic.LIF["g_ui"]
    template = synthetic.whole_brain(R=a.regions, mean_size=a.region_size, sigma=0.5, K=a.K, gen_seed=a.seed,
                                     g_ui=(g0[0] * a.gain, g0[1] * a.gain, g0[2], g0[3]),
                                     name=f"da_template_{a.regions}x{int(a.region_size)}")
    base = dict(steps_per_window=a.steps_per_window, seed=a.seed)
    rng = np.random.default_rng(a.seed + 99)

    # ---- truth and observations
    hp_true = torch.from_numpy(rng.uniform(0.6, 1.4, (template.R, 4)).astype(np.float32)).to(dev)
    obs = observe(template, hp_true, a.windows, base, a.seed + 5)

    def summarize(res, label):
        bp = res["bold_pred"][a.skip:]
        ob = obs.cpu().numpy()[a.skip:len(res["bold_pred"])]
        rmse = float(np.sqrt(np.mean((bp - ob) ** 2)))
        hp_fin = res["hp_mean"][-min(10, len(res["hp_mean"])):].mean(0)
        gerr = float(np.mean(np.abs(hp_fin - hp_true.cpu().numpy()) / hp_true.cpu().numpy()))
        ws = res["window_s"]
        return {f"{label}_window_s": float(np.mean(ws[1:] if len(ws) > 1 else ws)), f"{label}_rmse": rmse,
                f"{label}_gui_rel_err": gerr}

    out = dict(members=a.members, judges=a.judges, regions=a.regions, region_size=a.region_size, K=a.K, gain=a.gain,
               windows=a.windows, steps_per_window=a.steps_per_window,
               neurons_per_member=template.N, synapses_per_member=template.S)

    # ---- plain: every member on the simulator (first seed = the surrogate run's seed)
    plain_rmse = []
    for k in range(max(1, a.plain_seeds)):
        plain = EnsembleDA(template, DAConfig(n_members=a.members, **{**base, "seed": a.seed + 1000 * k}))
        res_k = plain.run(obs)
        sk = summarize(res_k, "plain")
        plain_rmse.append(sk["plain_rmse"])
        if k == 0:
            res_p = res_k
            out.update(sk)
        del plain
        torch.cuda.empty_cache()
    out["plain_rmse_by_seed"] = plain_rmse

    # ---- surrogate training windows: an assimilation run against another hidden truth, or a
    #      separate random-walk ensemble
    t0 = time.perf_counter()
    sets = []
    if a.train_source in ("da", "both"):
        hp_train = torch.from_numpy(np.random.default_rng(a.seed + 31).uniform(0.6, 1.4, (template.R, 4))
                                    .astype(np.float32)).to(dev)
        obs_train = observe(template, hp_train, a.train_windows, {**base, "seed": a.seed + 11}, a.seed + 13)
        sets.append(collect_da_windows(template, DAConfig(n_members=a.members, **{**base, "seed": a.seed + 7}),
                                       obs_train))
    if a.train_source in ("walk", "both"):
        sets.append(collect_windows(template, DAConfig(n_members=a.members, hp_sigma=a.train_sigma,
                                                       **{**base, "seed": a.seed + 17}), windows=a.train_windows))
    g, h, tgt = (torch.cat([x[i] for x in sets]) for i in range(3))
    t_collect = time.perf_counter() - t0
    n = g.shape[0]
    perm = torch.from_numpy(np.random.default_rng(a.seed).permutation(n))
    ntr = int(0.9 * n)
    tr, te = perm[:ntr], perm[ntr:]
    sur = RateSurrogate(seed=a.seed)
    t0 = time.perf_counter()
    hist = sur.fit(g[tr], h[tr], tgt[tr], epochs=a.epochs)
    t_train = time.perf_counter() - t0
    pred = sur.predict(g[te], h[te]).cpu()
    eps = 1e-6
    lerr_net = float(torch.sqrt(torch.mean((torch.log(pred + eps) - torch.log(tgt[te] + eps)) ** 2)))
    lerr_persist = float(torch.sqrt(torch.mean((torch.log(h[te][:, HISTORY - 1] + eps) - torch.log(tgt[te] + eps)) ** 2)))
    val_err = judge_error(pred, tgt[te])
    threshold = a.threshold if a.threshold is not None else a.margin * val_err
    out.update(heldout_judge_err=val_err, threshold=threshold)
    out.update(train_samples=int(n), train_windows=a.train_windows, train_source=a.train_source, train_sigma=a.train_sigma,
               train_collect_s=t_collect, train_s=t_train,
               train_loss_first=hist[0], train_loss_last=hist[-1], heldout_logrmse_net=lerr_net,
               heldout_logrmse_persistence=lerr_persist)

    # ---- surrogate-served DA
    sda = SurrogateDA(template, DAConfig(n_members=a.members, **base), sur, n_judge=a.judges,
                      threshold=threshold, adapt_steps=a.adapt_steps, bias_correct=bool(a.bias_correct),
                      spread=bool(a.spread), adapt_split=bool(a.adapt_split), self_history=bool(a.self_history))
    sda.hp_random_initialize()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    sda.burn_in(a.burn_in_windows)
    torch.cuda.synchronize(dev)
    t_burn = time.perf_counter() - t0
    res_s = sda.run(obs)
    out.update(summarize(res_s, "surrogate"))
    out.update(fallbacks=int(res_s["fallbacks"]), judge_err_mean=float(np.mean(res_s["errors"])),
               judge_err=[round(float(e), 4) for e in res_s["errors"]], adapt_steps=a.adapt_steps, adapt_split=a.adapt_split, self_history=a.self_history,
               bias_correct=a.bias_correct, spread=a.spread)
    out["surrogate_burn_in_s"] = t_burn
    out["burn_in_windows"] = a.burn_in_windows
    out["plain_total_s"] = float(np.sum(res_p["window_s"]))
    out["surrogate_total_s"] = float(np.sum(res_s["window_s"])) + t_burn
    out["speedup_total"] = out["plain_total_s"] / out["surrogate_total_s"]
    out["speedup"] = out["plain_window_s"] / out["surrogate_window_s"]
    out["rmse_ratio"] = out["surrogate_rmse"] / out["plain_rmse"]
    # windows served by the surrogate (no fallback), after the first
    fb = np.array(res_s["errors"]) > threshold
    ws = np.array(res_s["window_s"])
    served = [w for i, w in enumerate(ws) if i > 0 and not fb[i]]
    if served:
        out["surrogate_served_window_s"] = float(np.mean(served))
        out["speedup_served_windows"] = out["plain_window_s"] / out["surrogate_served_window_s"]
    out["plain_rmse_seed_spread"] = float(np.max(plain_rmse) / np.min(plain_rmse) - 1.0) if len(plain_rmse) > 1 else None
    out["total_s"] = time.perf_counter() - t_all
    line = json.dumps(out)
    if not quiet:
        print(line)
    if a.out:
        with open(a.out, "w") as f:
            f.write(line + "\n")
    return out


if __name__ == "__main__":
    main()
