"""Generate the golden fixtures from the reference's own Python code.

Runs only where a checkout of the reference is available, named by
$DTB_REFERENCE.  For each case it writes the network in
the reference's block_{i}.npz layout, loads it with the reference's
generation/read_block.py:connect_for_block, and steps the reference's
models/block.py:block with torch.rand replaced by the Philox4x32-10 noise
stream (oracle/philox layout), recording the per-step results.  The BOLD
fixture runs models/bold_model_pytorch.py:BOLD directly.

    DTB_REFERENCE=/path/to/Digital_twin_brain python tests/golden/make_golden.py

Outputs (committed): tests/golden/*.npz and tests/golden/small_blocks/.
"""
from __future__ import annotations

import os
import shutil
import sys
import tempfile

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("DTB_REFERENCE")   # the reference checkout (yeyeleijun/Digital_twin_brain)
if not REF or not os.path.isdir(REF):
    sys.exit("set DTB_REFERENCE to a checkout of the reference, e.g. DTB_REFERENCE=/path/to/Digital_twin_brain python tests/golden/make_golden.py")
sys.path.insert(0, ROOT)
sys.path.insert(0, REF)

from oracle import oracle as O  # noqa: E402
from digital_twin_brain_b200 import synthetic  # noqa: E402
from digital_twin_brain_b200.generation import write_blocks  # noqa: E402
from generation.read_block import connect_for_block  # noqa: E402  (reference)
from models.block import block as RefBlock  # noqa: E402  (reference)
from models.bold_model_pytorch import BOLD as RefBOLD  # noqa: E402  (reference)
from default_params import bold_params  # noqa: E402  (reference)


class PhiloxRand:
    """Stand-in for torch.rand(N): the Philox noise stream, one call per step."""

    def __init__(self, seed: int):
        self.seed = seed
        self.step = 0
        self.orig = torch.rand

    def __call__(self, *size, device=None, **kw):
        n = int(np.prod(size[0] if isinstance(size[0], (tuple, list)) else size))
        u = O.noise_uniforms_numpy(self.seed, self.step, n)
        self.step += 1
        return torch.from_numpy(u)

    def __enter__(self):
        torch.rand = self
        return self

    def __exit__(self, *a):
        torch.rand = self.orig


def packbits(b: np.ndarray) -> np.ndarray:
    return np.packbits(np.asarray(b, bool), axis=-1, bitorder="little")


def run_reference(dirpath: str, dt: float, seed: int, schedule, record_v_every: int, prop_update=None):
    """schedule: list of (n_steps, noise_rate, isolated). prop_update: (step, new_property) or None."""
    prop, W = connect_for_block(dirpath)
    b = RefBlock(prop, W, delta_t=dt)
    out = {k: [] for k in ("active", "new_active", "sums", "means", "V")}
    k = 0
    with PhiloxRand(seed) as rnd:
        for n, rate, iso in schedule:
            for _ in range(n):
                if prop_update is not None and k == prop_update[0]:
                    b.update_property(torch.from_numpy(prop_update[1]))
                s, m = b.run(noise_rate=rate, isolated=iso)
                # new_active is not kept by the reference; recompute it from the same stream
                u = O.noise_uniforms_numpy(seed, k, prop.shape[0])
                noise = u < np.float32(rate)
                na = noise if iso else (noise | b.active.numpy())
                out["active"].append(packbits(b.active.numpy()))
                out["new_active"].append(packbits(na))
                out["sums"].append(s.numpy().astype(np.float32))
                out["means"].append(m.numpy().astype(np.float32))
                if (k + 1) % record_v_every == 0:
                    out["V"].append(b.V_i.numpy().copy())
                k += 1
        assert rnd.step == k
    res = {key: np.stack(v) for key, v in out.items()}
    res.update(V_final=b.V_i.numpy(), J_final=b.J_ui.numpy(), I_ui_final=b.I_ui.numpy(),
               I_syn_final=b.I_syn.numpy(), t_last_final=b.t_ik_last.numpy(), t_final=np.float32(b.t.item()))
    return prop.numpy(), res


def case_single_block(steps: int = 400):
    spec = synthetic.config_single_block()
    rowptr, pre, kind, w = O.gen_network(spec.as_dict())
    N = spec.N
    post = np.repeat(np.arange(N), spec.K)
    prop = spec.property()
    bounds = [0, int(spec.region_n_exc[0]), N]
    tmp = tempfile.mkdtemp()
    try:
        write_blocks(tmp, prop, bounds, post, pre.astype(np.int64), kind, w)
        ref_prop, res = run_reference(tmp, spec.dt, spec.seed, [(steps, 0.01, False)], record_v_every=50)
    finally:
        shutil.rmtree(tmp)
    assert np.array_equal(ref_prop, prop)
    np.savez_compressed(os.path.join(HERE, "single_block_2k.npz"), steps=steps, seed=spec.seed, dt=spec.dt,
                        noise_rate=0.01, v_every=50, **res)
    print("single_block_2k: mean spikes/step", res["sums"].sum(1).mean(), "nact/step",
          np.unpackbits(res["new_active"], axis=-1, bitorder="little").sum(1).mean())


def case_small_unsorted(seed: int = 7):
    """N=300 in 3 populations, per-neuron random parameters, rows in random file order,
    a noise/isolation schedule and one update_property call."""
    rng = np.random.default_rng(seed)
    sizes = [150, 100, 50]
    bounds = np.concatenate([[0], np.cumsum(sizes)])
    N = int(bounds[-1])
    K = 30
    rows = []
    for i in range(N):
        src = rng.choice(N, K, replace=False)
        rows.append(src)
    post = np.repeat(np.arange(N), K)
    pre = np.concatenate(rows)  # random order inside each row
    pop_pre = np.searchsorted(bounds, pre, side="right") - 1
    kind = np.where(pop_pre == 2, 2, 0).astype(np.uint8)
    w = (rng.random((N * K, 2)) * 2.0).astype(np.float32)
    prop = np.zeros((N, 22), np.float32)
    pop = np.searchsorted(bounds, np.arange(N), side="right") - 1
    prop[:, 0] = 0.01
    prop[:, 2] = rng.uniform(0.0, 0.5, N)
    prop[:, 3] = pop
    prop[:, 4] = rng.uniform(0.5, 1.5, N)
    prop[:, 5] = rng.choice([2.0, 5.0], N)
    prop[:, 6] = rng.uniform(0.02, 0.04, N)
    prop[:, 7] = -70.0
    prop[:, 8] = -50.0
    prop[:, 9] = rng.choice([-55.0, -60.0], N)
    prop[:, 10:14] = rng.uniform(0.5, 1.5, (N, 4)) * np.array([0.01, 0.0005, 0.1, 0.005])
    prop[:, 14:18] = (0.0, 0.0, -70.0, -100.0)
    prop[:, 18:22] = rng.choice([2.0, 8.0], (N, 1)) * np.array([1.0, 20.0, 5.0, 25.0]) / 2.0
    prop = prop.astype(np.float32)
    new_prop = prop.copy()
    new_prop[:, 10:14] *= np.float32(1.3)
    new_prop[:, 2] = 0.0
    d = os.path.join(HERE, "small_blocks")
    if os.path.isdir(d):
        shutil.rmtree(d)
    write_blocks(d, prop, bounds, post, pre, kind, w)
    schedule = [(120, 0.01, False), (40, 0.02, True), (140, 0.005, False)]
    ref_prop, res = run_reference(d, 0.1, 11, schedule, record_v_every=1, prop_update=(200, new_prop))
    assert np.array_equal(ref_prop, prop)
    np.savez_compressed(os.path.join(HERE, "small_blocks_ref.npz"), seed=11, dt=0.1,
                        schedule=np.array(schedule, dtype=np.float64), update_step=200, new_property=new_prop,
                        **res)
    print("small_blocks: mean spikes/step", res["sums"].sum(1).mean())


def case_src(seed: int = 13, steps: int = 150):
    """Input neurons (models/block.py:37-50, :104-109): N=200, neurons 0..39 have no incoming
    synapse and replay a raster of steps + 1 columns."""
    rng = np.random.default_rng(seed)
    N, n_src, K = 200, 40, 20
    post = np.repeat(np.arange(n_src, N), K)
    pre = np.concatenate([rng.choice(N, K, replace=False) for _ in range(n_src, N)])
    kind = np.where(pre >= 160, 2, 0).astype(np.uint8)
    w = (rng.random((len(post), 2)) * 2.0).astype(np.float32)
    spec = synthetic.config_single_block()
    prop = np.repeat(spec.class_property[:1], N, axis=0).copy()
    prop[160:] = spec.class_property[1]
    prop[:, 3] = np.where(np.arange(N) < n_src, 0, np.where(np.arange(N) < 160, 1, 2))
    prop[:, 2] = rng.uniform(0.0, 0.6, N)
    prop[:, 10:14] *= np.float32(3.0)
    prop = prop.astype(np.float32)
    src = rng.random((n_src, steps + 1)) < 0.08
    idx = np.stack([kind.astype(np.int64), post, pre])
    idx = np.stack([idx, idx], axis=-1)
    idx[0, :, 1] += 1
    W = torch.sparse_coo_tensor(torch.from_numpy(idx.reshape(3, -1)), torch.from_numpy(w.reshape(-1).copy()),
                                (4, N, N))
    b = RefBlock(torch.from_numpy(prop), W, delta_t=0.1, src=torch.from_numpy(src))
    assert np.array_equal(b.src_neuron.numpy(), np.arange(n_src))
    out = {k: [] for k in ("active", "sums", "means", "V")}
    with PhiloxRand(0) as rnd:
        for _ in range(steps):
            sm, m = b.run(noise_rate=0.01)
            out["active"].append(packbits(b.active.numpy()))
            out["sums"].append(sm.numpy().astype(np.float32))
            out["means"].append(m.numpy().astype(np.float32))
            out["V"].append(b.V_i.numpy().copy())
        try:
            b.run(noise_rate=0.01)
            raise AssertionError("the reference accepted a step past its raster")
        except IndexError:
            pass
        assert rnd.step == steps     # the failing step raises before drawing its noise
    res = {key: np.stack(v) for key, v in out.items()}
    np.savez_compressed(os.path.join(HERE, "src_block_ref.npz"), prop=prop, post=post, pre=pre, kind=kind, w=w,
                        src=src, seed=0, dt=0.1, steps=steps, J_final=b.J_ui.numpy(), I_syn_final=b.I_syn.numpy(),
                        t_last_final=b.t_ik_last.numpy(), **res)
    act = np.unpackbits(res["active"], axis=-1, bitorder="little")[:, :N]
    print("src_block: input spikes/step", act[:, :n_src].sum(1).mean(), "others", act[:, n_src:].sum(1).mean())


def case_bold(steps: int = 300, R: int = 16, seed: int = 3):
    rng = np.random.default_rng(seed)
    out = {}
    for name, dt in (("f32", torch.float32), ("f64", torch.float64)):
        us = rng.uniform(0.0, 0.05, (steps, R))
        m = RefBOLD(**bold_params, delta_t=1e-4)
        outs = []
        for k in range(steps):
            outs.append(m.run(torch.from_numpy(us[k]).to(dt)).numpy())
        out[f"u_{name}"] = us
        out[f"bold_{name}"] = np.stack(outs)
        for f in ("s", "q", "v", "f_in"):
            out[f"{f}_{name}"] = getattr(m, f).numpy()
    # state_update then 20 steps (float32)
    w = rng.uniform(0.0, 1.5, (2, R // 2, 6)).astype(np.float32)
    w[0, 0, 1] = -1.0  # clamped to 1e-5
    m = RefBOLD(**bold_params, delta_t=1e-4)
    m.state_update(torch.from_numpy(w))
    us = rng.uniform(0.0, 0.05, (20, R)).astype(np.float32)
    outs = [m.run(torch.from_numpy(us[k])).numpy() for k in range(20)]
    out.update(su_w=w, su_u=us, su_bold=np.stack(outs))
    np.savez_compressed(os.path.join(HERE, "bold_ref.npz"), delta_t=1e-4, **out)
    print("bold: ok")


def case_enkf(seed: int = 5):
    """data_assimilation/DataAssimilation.py:40-60 diffusion_enkf with torch.normal fixed."""
    sys.path.insert(0, os.path.join(REF, "data_assimilation"))
    import importlib.util
    spec = importlib.util.spec_from_file_location("ref_da_enkf", os.path.join(REF, "data_assimilation",
                                                                              "DataAssimilation.py"))
    src = open(spec.origin).read()
    # only the filter function: the module imports matplotlib and the gRPC simulation at top level
    start = src.index("def diffusion_enkf(")
    end = src.index("class DataAssimilation(")
    ns = {"torch": torch, "np": np}
    exec(compile(src[start:end], spec.origin, "exec"), ns)
    rng = np.random.default_rng(seed)
    out = {}
    for name, (E, R, S) in {"small": (8, 5, 10), "da": (128, 90, 10)}.items():
        w_hat = torch.from_numpy(rng.normal(0.0, 1.0, (E, R, S)).astype(np.float32))
        w_hat[:, :, -1] = torch.from_numpy(rng.uniform(0.01, 0.05, (E, R)).astype(np.float32))
        bold_t = torch.from_numpy(rng.uniform(0.01, 0.05, (1, R)).astype(np.float32))
        noise = torch.from_numpy(rng.normal(0.0, 1.0, (E, R)).astype(np.float32))
        orig = torch.normal
        torch.normal = lambda *a, **k: noise.clone()
        try:
            w = ns["diffusion_enkf"](w_hat, 1e-4, bold_t, 0.8)
        finally:
            torch.normal = orig
        out.update({f"{name}_w_hat": w_hat.numpy(), f"{name}_bold_t": bold_t.numpy(), f"{name}_noise": noise.numpy(),
                    f"{name}_w": w.numpy()})
    np.savez_compressed(os.path.join(HERE, "enkf_ref.npz"), bold_sigma=1e-4, solo_rate=0.8, **out)
    print("enkf: ok")


def case_statistics(seed: int = 9):
    """analysis/spike_statistics.py and analysis/getpsd.py on a random raster (matplotlib stubbed:
    the module imports it at top level and it is not installed here)."""
    import types
    sys.modules.setdefault("matplotlib", types.ModuleType("matplotlib"))
    sys.modules.setdefault("matplotlib.pyplot", types.ModuleType("matplotlib.pyplot"))
    import numpy as _np
    if not hasattr(_np, "int"):
        _np.int = int      # analysis/getpsd.py:10 uses np.int, removed from numpy
    from analysis import spike_statistics as S
    from analysis import getpsd as G
    rng = np.random.default_rng(seed)
    p = rng.uniform(0.0005, 0.02, 60)
    raster = (rng.random((5000, 60)) < p).astype(np.uint8)
    f, pw = S.spike_psd(raster)
    sig = rng.normal(0, 1, 6000)
    gf, gp = G.get_psd(sig, fs=1000, resolution=0.5)
    np.savez_compressed(os.path.join(HERE, "statistics_ref.npz"), raster=raster, rate=S.mean_firing_rate(raster),
                        inst=S.instantaneous_rate(raster), cv=S.coefficient_of_variation(raster), psd_f=f, psd=pw,
                        sig=sig, welch_f=gf, welch=gp)
    print("statistics: ok")


if __name__ == "__main__":
    torch.set_num_threads(8)
    if "--src" in sys.argv:
        case_src()
        sys.exit(0)
    if "--statistics" in sys.argv:
        case_statistics()
        sys.exit(0)
    if "--enkf" in sys.argv:
        case_enkf()
        sys.exit(0)
    case_bold()
    case_small_unsorted()
    case_single_block()
