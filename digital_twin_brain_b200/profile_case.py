"""A small, self-ending case of the step kernels for profilers.

    python -m digital_twin_brain_b200.profile_case [--scale S] [--K K] [--steps n] [--mode push|pull]

Builds the whole-brain network structure at `scale` with in-degree K (the
defaults keep J and the state above the 126 MB L2 while the synapse tables
stay at a few GB), runs a short warm-up and then `steps` steps with one
kernel launch per stage (no CUDA graphs), so a profiler can select single
launches of k_step / k_scatter.
"""
from __future__ import annotations

import argparse

import torch

from . import Network, synthetic
from ._lib import TUNE_J_CACHE, TUNE_SCATTER_WORDS, TUNE_STEP_VARIANT, TUNE_USE_GRAPHS


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scale", type=float, default=0.45)
    ap.add_argument("--K", type=int, default=20)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=80)
    ap.add_argument("--mode", default="push", choices=["push", "pull"])
    ap.add_argument("--scatter-words", type=int, default=0)
    ap.add_argument("--step-variant", type=int, default=0, help="0/1: register budgets, 2/3/4: staged state loads (2, 3, 4 CTAs per SM)")
    ap.add_argument("--j-cache", type=int, default=0, help="1: the update's J stores keep their L2 lines")
    a = ap.parse_args()
    spec = synthetic.whole_brain(K=a.K, scale=a.scale, name="profile_case")
    net = Network.from_spec(spec, device=0, build_push=True)   # pull runs as the ordered push
    net.set_tuning(TUNE_USE_GRAPHS, 0)
    net.set_tuning(TUNE_STEP_VARIANT, a.step_variant)
    net.set_tuning(TUNE_J_CACHE, a.j_cache)
    if a.scatter_words:
        net.set_tuning(TUNE_SCATTER_WORDS, a.scatter_words)
    net.run(a.warmup, mode=a.mode, out=None)
    torch.cuda.synchronize()
    t = net.time_kernels(a.steps, mode=a.mode)
    info = net.info()
    print(f"profile_case N={spec.N} S={spec.S} device_GB={info.device_bytes / 1e9:.2f} mode={a.mode} "
          f"step_variant={a.step_variant} j_cache={a.j_cache} {t}")


if __name__ == "__main__":
    main()
