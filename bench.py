"""Benchmark of the Digital Twin Brain time-step path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one dt = 0.1 ms time step of the whole-brain workload: 90 regions
of log-normal size (~2.2e7 neurons), K = 100 presynaptic neurons each
(~2.2e9 synapses), 80 % intra-region, Poisson noise p = 0.01, per-region
Balloon-Windkessel BOLD.  Synthetic network (seeded), since the reference's
imaging-derived inputs are not available.

value = synaptic events/s (sum over steps of the out-degrees of every neuron
that propagated, i.e. spike | noise, divided by device time), timed with CUDA
events on the network's stream over exactly K steps after W warm-up steps,
max over ranks.  The state (1 GB) and synapse tables (27 GB per direction)
are far larger than L2, so no flush is needed.  With N GPUs every rank runs
an independent replica (the path does not shard across GPUs).

--impl reference times the reference's algorithm on the host cores (the CPU
oracle restating models/block.py, OpenMP) on a bounded sample of the same
workload and prints the same line with "impl": "reference".

Other workloads (--config): one_region (N=1e6, K=100; --noise sweeps the pull/push
crossover), single_block (N=2000), ensemble (64 members of U[5e4,4e5] neurons with
per-member g_ui, one BOLD region each) and profile_case (the whole-brain structure
at scale 0.45 with K=20: a few GB on the device, the case the ncu captures use).
The default whole-brain run also runs the data-assimilation comparison (surrogate-
served vs all-simulator ensemble, digital_twin_brain_b200/da_bench.py) at a
reduced region size and reports it under "da".
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "synaptic events/s & sim-s/wall-s at 2B syn; DA window time surrogate vs plain"
UNIT = "events/s"
# DRAM traffic per unit processed, from ncu captures (dram__bytes_read.sum + dram__bytes_write.sum)
# of single launches: the atomic push scatter per synaptic event and the staged update per neuron.
# The line's roofline.traffic scales these to the launch it reports and says so.
SCATTER_DRAM_BYTES_PER_EVENT = (943.26e6 + 360.44e6) / 23462598
UPDATE_DRAM_BYTES_PER_NEURON = (595.12e6 + 418.77e6) / 23448955


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--warmup", type=int, default=200)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--mode", default="tune", choices=["tune", "auto", "push", "pull"])
    ap.add_argument("--scale", type=float, default=1.0, help="whole-brain size scale (1.0 = ~2.2e9 synapses)")
    ap.add_argument("--config", default="whole_brain",
                    choices=["whole_brain", "one_region", "single_block", "ensemble", "profile_case"],
                    help="whole_brain: 90 regions ~2.2e9 synapses (the headline); one_region: N=1e6, K=100; "
                         "single_block: N=2000, K=100; ensemble: 64 members N~U[5e4,4e5], per-member g_ui; "
                         "profile_case: whole-brain structure x0.45, K=20 (ncu captures)")
    ap.add_argument("--noise", type=float, default=0.01)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=400)
    ap.add_argument("--graphs", type=int, default=1, help="0: one launch per kernel (profilers)")
    ap.add_argument("--push-method", type=int, default=-1, help="1 atomics, 2 binned (-1: autotuned / default)")
    ap.add_argument("--pull-method", type=int, default=-1, help="1 rows, 2 slots, 3 masks, 4 streamed (-1: auto)")
    ap.add_argument("--step-variant", type=int, default=-1, help="update kernel variant 0..4 (-1: autotuned)")
    ap.add_argument("--scatter-words", type=int, default=0, help="atomic scatter bitmask words per warp (0: tuned)")
    ap.add_argument("--da", type=int, default=-1,
                    help="1: run the data-assimilation comparison (default: on for the whole-brain line)")
    ap.add_argument("--da-region-size", type=float, default=2000)
    ap.add_argument("--da-windows", type=int, default=24)
    ap.add_argument("--da-members", type=int, default=128)
    ap.add_argument("--da-train-windows", type=int, default=10)
    return ap.parse_args()


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 50 ms, from the kernel timing through
    the timed region to the end-to-end run."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = self.smi_id(gpu_index)
        self.proc = None
        self.lines = []

    @staticmethod
    def smi_id(dev: int) -> str:
        """nvidia-smi's name for CUDA device `dev`: its UUID when nvidia-smi answers to it (CUDA's
        device order need not be nvidia-smi's index order), else the index."""
        try:
            import torch
            u = str(torch.cuda.get_device_properties(dev).uuid)
            u = u if u.startswith("GPU-") else "GPU-" + u
            r = subprocess.run(["nvidia-smi", "--query-gpu=uuid", "--format=csv,noheader", "-i", u],
                               capture_output=True, text=True, timeout=20)
            if r.returncode == 0 and r.stdout.strip().lower() == u.lower():
                return u
        except Exception:
            pass
        return str(dev)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", self.gpu, "-lms", "50"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"), f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


def combine_over_ranks(ms: float, events: float, world: int, device) -> tuple:
    """Whole-job figures of N replicas: the slowest rank's device time, the events of all ranks."""
    if world <= 1:
        return ms, events
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms, events], dtype=torch.float64, device=device)
    mx = t.clone()
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    tot = t.clone()
    dist.all_reduce(tot, op=dist.ReduceOp.SUM)
    return float(mx[0]), float(tot[1])


# ---------------------------------------------------------------- CPU baseline
def cpu_sample(scale: float, noise: float, seconds: float, max_steps: int, warmup: int = 2):
    """The reference algorithm (oracle port of models/block.py, OpenMP) on a scaled whole-brain network."""
    from oracle import oracle as O
    from digital_twin_brain_b200 import synthetic
    import torch
    threads = min(os.cpu_count() or 1, 64)
    spec = synthetic.whole_brain(scale=scale, noise_rate=noise, name="cpu_sample")
    rowptr, pre, kind, w = O.gen_network(spec.as_dict())
    prop = spec.property()
    tau = torch.from_numpy(prop).transpose(0, 1)[18:22]
    decay = torch.exp(-spec.dt / tau).numpy().copy()
    ob = O.OracleBlock(prop, decay, rowptr, pre, kind, w, spec.dt, spec.seed, nthreads=threads)
    outdeg = np.bincount(pre, minlength=spec.N).astype(np.int64)
    for _ in range(warmup):
        ob.run(noise)
    events = 0
    steps = 0
    t0 = time.perf_counter()
    while steps < max_steps and (time.perf_counter() - t0) < seconds:
        ob.run(noise)
        events += int(outdeg[ob.new_active.astype(bool)].sum())
        steps += 1
    dt = time.perf_counter() - t0
    return dict(value=events / dt, unit=UNIT, cores=threads, kind="port", steps=steps, seconds=dt,
                sim_s_per_wall_s=steps * spec.dt / 1000.0 / dt,
                sample=(f"oracle port of models/block.py step (sparse gather over all {spec.S} synapses, "
                        f"{threads} OpenMP threads) on the whole-brain network at scale {scale}: "
                        f"N={spec.N}, S={spec.S}, {steps} steps after {warmup} warm-up"))


# ---------------------------------------------------------------- reference arm
def run_reference(args, rank: int, world: int):
    if rank != 0:
        return
    budget = 60.0
    r = cpu_sample(scale=1 / 64, noise=args.noise, seconds=budget, max_steps=max(args.steps, 1),
                   warmup=min(args.warmup, 3))
    line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": r["steps"],
            "warmup": min(args.warmup, 3), "ms_per_step": 1000.0 * r["seconds"] / max(r["steps"], 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": "whole_brain_90 (90 regions, K=100, dt=0.1 ms, p=0.01) at scale 1/64 on CPU",
                       "parallelism": "host cores"},
            "sim_s_per_wall_s": r["sim_s_per_wall_s"],
            "cpu_baseline": {"value": r["value"], "unit": UNIT, "cores": r["cores"], "kind": r["kind"],
                             "sample": r["sample"]},
            "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ---------------------------------------------------------------- our arm
def build_spec(args, rank: int):
    from digital_twin_brain_b200 import synthetic
    if args.config == "one_region":
        spec = synthetic.config_one_region(args.noise)
    elif args.config == "single_block":
        spec = synthetic.config_single_block()
    elif args.config == "ensemble":
        spec = synthetic.config_ensemble(scale=args.scale)
    elif args.config == "profile_case":
        spec = synthetic.whole_brain(K=20, scale=0.45, name="profile_case_wb90_x0.45_K20")
    else:
        spec = synthetic.config_whole_brain(args.scale) if args.scale != 1.0 else synthetic.config_whole_brain()
    spec.seed = 1000 + rank              # independent replica noise per rank
    spec.extra["noise"] = args.noise
    return spec


def describe(spec, args) -> str:
    N, S = spec.N, spec.S
    if args.config == "ensemble":
        sizes = spec.extra["member_sizes"]
        return (f"{spec.name}: {len(sizes)} members of N~U[5e4,4e5] x{args.scale} ({min(sizes)}..{max(sizes)}), "
                f"N={N}, S={S}, K={spec.K}, per-member g_ui x U[0.5,1.5], dt=0.1 ms, noise p={args.noise}, "
                f"fp32 weights, BOLD per member")
    if args.config in ("one_region", "single_block"):
        return f"{spec.name}: one region, N={N}, S={S}, K={spec.K}, 80/20 E/I, dt=0.1 ms, noise p={args.noise}, fp32 weights"
    sc = " x0.45" if args.config == "profile_case" else (f" x{args.scale}" if args.scale != 1.0 else "")
    return (f"{spec.name}: {spec.R} regions lognormal(ln 2.2e5, 0.5){sc}, N={N}, S={S}, K={spec.K}, "
            f"80% intra-region, dt=0.1 ms, noise p={args.noise}, fp32 weights, BOLD per region")


def roofline_of(spec, kt, mode, push_method, pull_method, peaks):
    """Algorithmic bytes of every kernel of the step (per launch) and the dominant kernel's roofline."""
    N, S = spec.N, spec.S
    evs = kt["events_per_step"]
    nact = evs / spec.K
    # V, J, t_last read, one class id per 128-neuron tile; V, J written; two bitmasks
    upd_bytes = N * (4 + 16 + 4 + 4 / 128) + N * (4 + 16) + 2 * N / 8
    prop_bytes = N / 8 + 16 * nact + 12 * evs                              # bitmask, row pointers, (post, w) of rows
    # pull mode runs as ordered push with method 2 (slots) or 3 (masks), or when auto (0) picks
    # slots at low activity (active fraction <= 0.1); rows (1) and streamed (4) are one fused kernel
    ordered = mode == "pull" and (pull_method in (2, 3) or (pull_method in (0, -1) and nact / N <= 0.1))
    if mode == "push" and push_method == 2:
        # binned: the scatter also writes every event into its bin (u16 index + weight pair), the
        # update reads them back
        kernels = {"update+fold": (kt["update_ms"], upd_bytes + 10 * evs),
                   "binned scatter": (kt["propagate_ms"], prop_bytes + 10 * evs)}
    elif mode == "push":
        kernels = {"update": (kt["update_ms"], upd_bytes), "scatter": (kt["propagate_ms"], prop_bytes)}
    elif ordered:
        # ordered push: + pull-row positions, slot writes; the update reads counts and slots
        kernels = {"slots+update": (kt["update_ms"], upd_bytes + 4 * N + 16 * evs),
                   "ordered scatter": (kt["propagate_ms"], prop_bytes + 2 * evs + 16 * evs)}
    else:
        fused = upd_bytes + 8 * N + 4 * S + 8 * evs                        # + row ptrs, all indices, active weights
        kernels = {"gather+update": (kt["update_ms"], fused)}
    dom = max(kernels, key=lambda k: kernels[k][0])
    d_ms, d_bytes = kernels[dom]
    peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved = d_bytes / (d_ms * 1e-3) / 1e9 if d_ms > 0 else 0.0
    traffic, tsrc = None, None
    if dom == "scatter":
        traffic = SCATTER_DRAM_BYTES_PER_EVENT * evs
        tsrc = "ncu DRAM bytes per synaptic event of the atomic scatter, scaled to this launch's events"
    elif dom == "update":
        traffic = UPDATE_DRAM_BYTES_PER_NEURON * N
        tsrc = "ncu DRAM bytes per neuron of the staged update, scaled to this launch's neurons"
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "traffic_source": tsrc, "kernel": dom, "algorithmic_bytes_per_launch": d_bytes,
                "launch_ms": d_ms,
                "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback 6650 GB/s"}
    per_kernel = {k: {"ms": v[0], "bytes": v[1], "gbs": v[1] / (v[0] * 1e-3) / 1e9 if v[0] > 0 else 0.0,
                      "frac": (v[1] / (v[0] * 1e-3) / 1e9) / peak if v[0] > 0 else 0.0} for k, v in kernels.items()}
    # the step against the reference layout's byte model: N*44 + S_touched*13 + N/8 per step
    model_bytes = N * 44 + evs * 13 + N / 8
    step = {"bytes_per_step_model": model_bytes, "ms": kt["step_ms"],
            "achieved_gbs": model_bytes / (kt["step_ms"] * 1e-3) / 1e9 if kt["step_ms"] else 0,
            "frac": (model_bytes / (kt["step_ms"] * 1e-3) / 1e9) / peak if kt["step_ms"] else 0,
            "kernels": per_kernel}
    return roofline, step


def atomic_probe(dev, N, evs, window):
    """float2 atomics per second on this GPU into J-sized targets (bench-only helper library)."""
    import ctypes
    from digital_twin_brain_b200 import build as B
    try:
        L = ctypes.CDLL(B.build_probe())
        fn = L.dtb_bench_atomic_rate
        fn.argtypes = [ctypes.c_int, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.POINTER(ctypes.c_float)]
        fn.restype = ctypes.c_int
        ms = ctypes.c_float()
        if fn(dev, int(N), int(max(evs, 1)), int(max(1, window)), ctypes.byref(ms)) != 0:
            return None
        return ms.value
    except Exception:
        return None


def mlp_measure(dev, peaks) -> dict:
    """The surrogate network's tensor-core kernels (tcgen05, BF16 operands, FP32 accumulation) timed
    on the DA forecast batch (128 members x 90 regions) and a training minibatch, against the
    measured dense BF16 peak.  Algorithmic FLOPs count each multiply-add of the network once (the
    kernels run three BF16 products per FP32 operand to keep FP32 accuracy).  `ms` is the device
    time of one call's kernels (the call captured once in a CUDA graph and replayed: no host time
    between launches); `ms_per_call` times the same calls issued one by one from Python."""
    import torch
    from digital_twin_brain_b200.surrogate import MLP
    torch.cuda.set_device(dev)
    in_dim, H = 14, 256
    m = MLP(in_dim, H, seed=0, device=dev)
    g = torch.Generator(device=f"cuda:{dev}").manual_seed(0)
    out = {}
    side = torch.cuda.Stream(device=dev)
    for name, B, fn in (("forward", 128 * 90, "fwd"), ("train_step", 4096, "train")):
        x = torch.randn(B, in_dim, device=f"cuda:{dev}", generator=g)
        t = torch.randn(B, device=f"cuda:{dev}", generator=g)
        run = (lambda: m.forward(x)) if fn == "fwd" else (lambda: m.train_step(x, t, 1e-4))
        for _ in range(3):
            run()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(20):
            run()
        e1.record()
        torch.cuda.synchronize(dev)
        ms_call = e0.elapsed_time(e1) / 20
        graph = torch.cuda.CUDAGraph()
        side.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(side):
            run()                                   # warm-up on the capture stream
            side.synchronize()
            with torch.cuda.graph(graph, stream=side):
                run()
        torch.cuda.synchronize(dev)
        for _ in range(3):
            graph.replay()
        torch.cuda.synchronize(dev)
        e0.record()
        for _ in range(50):
            graph.replay()
        e1.record()
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1) / 50
        del graph
        flops = 2.0 * B * (in_dim * H + H * H + H) * (1 if fn == "fwd" else 3)
        tf = flops / (ms * 1e-3) / 1e12
        peak = float(peaks.get("bf16_tflops", 1590.0))
        out[name] = {"rows": B, "ms": ms, "ms_per_call": ms_call, "tflops": tf, "peak_tflops": peak,
                     "frac": tf / peak, "unit": "TFLOP/s", "peak_source": "MEASURED_PEAKS.json bf16_tflops (of measured)"
                     if "bf16_tflops" in peaks else "fallback 1590 TFLOP/s"}
    m.close()
    return out


def run_da(args, dev):
    """The data-assimilation comparison (metric part 3) at a reduced region size."""
    from digital_twin_brain_b200 import da_bench
    argv = ["--members", str(args.da_members), "--judges", str(max(2, args.da_members // 16)),
            "--region-size", str(args.da_region_size), "--windows", str(args.da_windows),
            "--train-windows", str(args.da_train_windows), "--plain-seeds", "1", "--skip", "4"]
    r = da_bench.main(argv, quiet=True)
    keys = ("members", "judges", "regions", "region_size", "neurons_per_member", "windows", "steps_per_window",
            "plain_window_s", "surrogate_window_s", "speedup", "plain_total_s", "surrogate_total_s", "speedup_total",
            "surrogate_served_window_s", "speedup_served_windows", "fallbacks", "plain_rmse", "surrogate_rmse",
            "rmse_ratio", "plain_gui_rel_err", "surrogate_gui_rel_err", "train_windows", "train_samples",
            "train_collect_s", "train_s", "heldout_logrmse_net", "heldout_logrmse_persistence", "total_s")
    out = {k: r[k] for k in keys if k in r}
    out["note"] = ("surrogate_total_s includes its burn-in window; train_collect_s (simulating the training "
                   "windows) and train_s are outside both totals")
    return out


def run_ours(args, rank: int, world: int, local_rank: int):
    import torch
    import torch.distributed as dist
    from digital_twin_brain_b200 import Network
    from digital_twin_brain_b200._lib import (TUNE_PULL_METHOD, TUNE_PUSH_METHOD, TUNE_SCATTER_WORDS,
                                              TUNE_STEP_VARIANT, TUNE_USE_GRAPHS)

    dev = local_rank
    torch.cuda.set_device(dev)
    spec = build_spec(args, rank)
    t_build = time.perf_counter()
    net = Network.from_spec(spec, device=dev, build_push=True)
    bold_regions = spec.R
    net.attach_bold(spec.sub_to_region(), bold_regions, delta_t=spec.dt / 1000.0)
    stream = torch.cuda.Stream(device=dev)
    net.set_stream(stream)
    torch.cuda.synchronize(dev)
    t_build = time.perf_counter() - t_build
    info = net.info()
    if not args.graphs:
        net.set_tuning(TUNE_USE_GRAPHS, 0)

    # warm-up (also passes the initial refractory period) and method choice
    W = max(args.warmup, 3)
    net.run(W, noise_rate=args.noise, mode="auto", out=None)
    tune = {}
    if args.mode == "tune":
        tune = net.autotune(32, noise_rate=args.noise)
        mode = "push" if tune["push_ms"] <= tune["pull_ms"] else "pull"
    else:
        mode = args.mode
    if args.push_method >= 0:
        net.set_tuning(TUNE_PUSH_METHOD, args.push_method)
    if args.pull_method >= 0:
        net.set_tuning(TUNE_PULL_METHOD, args.pull_method)
    if args.step_variant >= 0:
        net.set_tuning(TUNE_STEP_VARIANT, args.step_variant)
    if args.scatter_words > 0:
        net.set_tuning(TUNE_SCATTER_WORDS, args.scatter_words)
    push_method = net.get_tuning(TUNE_PUSH_METHOD)
    pull_method = net.get_tuning(TUNE_PULL_METHOD)
    torch.cuda.synchronize(dev)

    clk = ClockSampler(dev)
    clk.__enter__()
    try:
        kt = net.time_kernels(64, noise_rate=args.noise, mode=mode)
        # the chunk graphs of the chosen method are captured here, outside the timed region
        net.run(64, noise_rate=args.noise, mode=mode, out=None)
        torch.cuda.synchronize(dev)

        # ---- timed region: exactly K steps on the device
        K = args.steps
        ev0 = net.get(10)  # FIELD_EVENTS
        l0 = net.info().kernel_launches
        start = torch.cuda.Event(enable_timing=True)
        end = torch.cuda.Event(enable_timing=True)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)
        start.record(stream)
        net.run(K, noise_rate=args.noise, mode=mode, out=None)
        end.record(stream)
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()
        ms = start.elapsed_time(end)
        events = net.get(10) - ev0
        launches = net.info().kernel_launches - l0
        ms_max, events_all = combine_over_ranks(ms, float(events), world, f"cuda:{dev}")
        value = events_all / (ms_max / 1000.0)
        sim_ratio = K * spec.dt / 1000.0 / (ms_max / 1000.0)

        # ---- end to end through the public API: per step, host->device run parameters and the
        #      per-subblock results (spike sums, mean V, propagated count) back to host memory
        E = min(args.e2e_steps, K)
        e2e = None
        if E > 0:
            ev_a = net.get(10)
            torch.cuda.synchronize(dev)
            if world > 1:
                dist.barrier()
            t0 = time.perf_counter()
            for _ in range(E):
                net.run(1, noise_rate=args.noise, mode=mode, out="host")
            t_e2e = time.perf_counter() - t0
            ev_e2e = net.get(10) - ev_a
            # whole job at N replicas: the events of all ranks over the slowest rank's time
            e2e_ms, ev_e2e = combine_over_ranks(1000.0 * t_e2e, float(ev_e2e), world, f"cuda:{dev}")
            t_e2e = e2e_ms / 1000.0
            h2d = 16                                  # run parameters (base step, noise rate, isolated)
            d2h = 2 * 4 * net.n_sub + 4               # spike sums + mean V per subblock + propagated count
            e2e = {"value": ev_e2e / t_e2e, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                   "steps": E, "ms_per_step": 1000.0 * t_e2e / E,
                   "api": "Network.run(1, out='host') per step (ctypes -> dtb_block_run, DTB_HOST)"}
    finally:
        clk.__exit__()

    # ---- roofline of the dominant kernel and of the step
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    roofline, step_roofline = roofline_of(spec, kt, mode, push_method, pull_method, peaks)

    # the atomic push scatter's own ceiling: float2 atomics per second on this GPU, measured live with
    # the same count into J-sized targets, destinations inside region-sized windows
    atomic = None
    evs = kt["events_per_step"]
    if mode == "push" and push_method != 2 and kt["propagate_ms"] > 0 and args.config != "profile_case":
        probe_ms = atomic_probe(dev, spec.N, evs, spec.N // spec.R)
        if probe_ms:
            peak_ops = evs / (probe_ms * 1e-3) / 1e9
            got_ops = evs / (kt["propagate_ms"] * 1e-3) / 1e9
            atomic = {"bound": "l2_atomics", "achieved": got_ops, "peak": peak_ops, "unit": "G float2 atomics/s",
                      "frac": got_ops / peak_ops, "kernel": "scatter",
                      "probe": f"dtb_bench_atomic_rate(N={spec.N}, ops={int(evs)}, window={spec.N // spec.R})"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.config in ("whole_brain",):
        r = cpu_sample(scale=1 / 64, noise=args.noise, seconds=15.0, max_steps=10_000)
        cpu = {"value": r["value"], "unit": UNIT, "cores": r["cores"], "kind": r["kind"], "sample": r["sample"]}

    da = None
    run_da_now = args.da == 1 or (args.da < 0 and args.config == "whole_brain" and args.scale == 1.0)
    if rank == 0 and world == 1 and run_da_now:
        net.close()
        net = None
        torch.cuda.empty_cache()
        da = run_da(args, dev)
        da["mlp"] = mlp_measure(dev, peaks)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
                "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic",
                "config": {"workload": describe(spec, args),
                           "method": mode + (("/binned" if push_method == 2 else "/atomic") if mode == "push" else ""),
                           "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                           "l2": "inputs larger than L2 (state ~1 GB, synapses ~27 GB per CSR)"
                                 if args.config == "whole_brain" else "inputs larger than L2"},
                "value_metric": "synaptic events/s", "sim_s_per_wall_s": sim_ratio,
                "events_per_step": events_all / world / K, "firing": {
                    "propagated_per_step": evs / spec.K, "propagated_frac": evs / spec.K / spec.N},
                "kernel_ms": kt, "tune": tune, "build_s": t_build, "device_gb": info.device_bytes / 1e9,
                "gpu_launches": int(launches),
                "roofline": roofline,
                "atomic_roofline": atomic,
                "step_roofline": step_roofline,
                "e2e": e2e,
                "clocks": clk.summary()}
        if cpu:
            line["cpu_baseline"] = cpu
        if da:
            line["da"] = da
        print(json.dumps(line))
    if net is not None:
        net.close()


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    import torch
    import torch.distributed as dist
    if world > 1:
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
