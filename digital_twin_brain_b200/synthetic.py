"""Seeded synthetic networks in the reference's layout.

The reference builds networks from brain-imaging data with
``generation/make_block.py`` (unseeded, ``make_block.py:677``); the data are
not available here, so these generators stand in for them with the shapes,
sizes and value distributions of the benchmark configurations:

* :func:`single_block` — one population pair (80 % excitatory), K random
  presynaptic neurons per neuron (the small-block recipe of
  ``test/test_generation.py:312-330`` with uniform sources);
* :func:`whole_brain` — regions of log-normal size, 80 % of the synapses
  inside the region and the rest routed by a seeded log-normal
  region-connectivity matrix.

A network is defined by a :class:`NetworkSpec`; the GPU generator
(``dtb_block_create_synthetic``) and the CPU oracle produce identical arrays
from it.  Property rows follow ``generation/make_block.py:394-432``.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

# LIF parameters of the single-block configuration (N=2000, K=100).
LIF = dict(noise_rate=0.01, I_extern_Input=0.0, C=1.0, T_ref=5.0, g_Li=0.03, V_L=-70.0, V_th=-50.0,
           V_reset=-55.0, g_ui=(0.01, 0.0005, 0.1, 0.005), V_ui=(0.0, 0.0, -70.0, -100.0),
           tao_ui=(2.0, 40.0, 10.0, 50.0))


def property_row(sub_block_idx: int, noise_rate=0.01, I_extern_Input=0.0, C=1.0, T_ref=5.0, g_Li=0.03,
                 V_L=-70.0, V_th=-50.0, V_reset=-55.0, g_ui=LIF["g_ui"], V_ui=LIF["V_ui"],
                 tao_ui=LIF["tao_ui"]) -> np.ndarray:
    """One row of the 22-column property matrix (generation/make_block.py:394-432)."""
    p = np.zeros(22, np.float32)
    p[0] = noise_rate
    p[1] = 0.0
    p[2] = I_extern_Input
    p[3] = sub_block_idx
    p[4] = C
    p[5] = T_ref
    p[6] = g_Li
    p[7] = V_L
    p[8] = V_th
    p[9] = V_reset
    p[10:14] = np.asarray(g_ui, np.float32)
    p[14:18] = np.asarray(V_ui, np.float32)
    p[18:22] = np.asarray(tao_ui, np.float32)
    return p


@dataclass
class NetworkSpec:
    name: str
    region_start: np.ndarray          # int64 [R+1]
    region_n_exc: np.ndarray          # int64 [R]
    cum: np.ndarray                   # float32 [R,R] cumulative source-region distribution
    K: int
    class_property: np.ndarray        # float32 [2R,22]; class 2r excitatory, 2r+1 inhibitory
    gen_seed: int = 0
    w_scale: float = 1.0
    dt: float = 0.1
    seed: int = 0                     # Philox noise key
    stream_id: int = 0
    members: dict | None = None       # ensemble tables (see ensemble()); None for one network
    extra: dict = field(default_factory=dict)

    @property
    def R(self) -> int:
        return len(self.region_start) - 1

    @property
    def N(self) -> int:
        return int(self.region_start[-1])

    @property
    def S(self) -> int:
        return self.N * self.K

    def as_dict(self) -> dict:
        d = dict(region_start=self.region_start, region_n_exc=self.region_n_exc, cum=self.cum, K=self.K,
                 gen_seed=self.gen_seed, w_scale=self.w_scale)
        if self.members is not None:
            d.update(self.members)
        return d

    def neuron_class(self) -> np.ndarray:
        """Class (= subblock) of every neuron: 2r excitatory, 2r+1 inhibitory."""
        cls = np.empty(self.N, np.int64)
        for r in range(self.R):
            s0, s1, ne = int(self.region_start[r]), int(self.region_start[r + 1]), int(self.region_n_exc[r])
            cls[s0:s0 + ne] = 2 * r
            cls[s0 + ne:s1] = 2 * r + 1
        return cls

    def property(self) -> np.ndarray:
        """Per-neuron [N,22] property matrix (subblock index in column 3)."""
        return self.class_property[self.neuron_class()].copy()

    def sub_to_region(self) -> np.ndarray:
        n_sub = int(self.class_property[:, 3].max()) + 1
        return (np.arange(n_sub) // 2).astype(np.int32)


def _classes(R: int, **lif) -> np.ndarray:
    return np.stack([property_row(c, **lif) for c in range(2 * R)])


def single_block(N: int = 2000, K: int = 100, exc_frac: float = 0.8, gen_seed: int = 0, seed: int = 0,
                 dt: float = 0.1, noise_rate: float = 0.01, name: str | None = None, **lif) -> NetworkSpec:
    """One region of N neurons (first exc_frac excitatory), K uniform distinct sources per neuron."""
    params = dict(LIF)
    params.update(lif)
    params["noise_rate"] = noise_rate
    return NetworkSpec(name=name or f"single_block_N{N}_K{K}",
                       region_start=np.array([0, N], np.int64),
                       region_n_exc=np.array([int(round(exc_frac * N))], np.int64),
                       cum=np.ones((1, 1), np.float32), K=K, class_property=_classes(1, **params),
                       gen_seed=gen_seed, seed=seed, dt=dt)


def whole_brain(R: int = 90, mean_size: float = 2.2e5, sigma: float = 0.5, K: int = 100, intra: float = 0.8,
                exc_frac: float = 0.8, gen_seed: int = 0, seed: int = 0, dt: float = 0.1,
                noise_rate: float = 0.01, scale: float = 1.0, name: str | None = None, **lif) -> NetworkSpec:
    """R regions of log-normal(ln mean_size, sigma) neurons (times `scale`), `intra` of the synapses inside
    the region, the rest routed by a seeded log-normal(0, 1) region matrix (row-normalised)."""
    rng = np.random.default_rng(gen_seed)
    sizes = np.maximum(np.round(rng.lognormal(np.log(mean_size), sigma, R) * scale), 2 * K + 2).astype(np.int64)
    M = rng.lognormal(0.0, 1.0, (R, R))
    np.fill_diagonal(M, 0.0)
    P = (1.0 - intra) * M / M.sum(axis=1, keepdims=True)
    P[np.arange(R), np.arange(R)] = intra
    cum = np.cumsum(P, axis=1)
    cum[:, -1] = 1.0
    params = dict(LIF)
    params.update(lif)
    params["noise_rate"] = noise_rate
    start = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    return NetworkSpec(name=name or f"whole_brain_R{R}", region_start=start,
                       region_n_exc=np.round(exc_frac * sizes).astype(np.int64), cum=cum.astype(np.float32), K=K,
                       class_property=_classes(R, **params), gen_seed=gen_seed, seed=seed, dt=dt)


def ensemble(templates: list, g_scale=None, stream_id: int = 0, name: str = "ensemble") -> NetworkSpec:
    """Members concatenated in one network (the data-assimilation ensemble layout of
    data_assimilation/DataAssimilation.py:97, members side by side in one block).

    Member m keeps its own regions, connectivity (synapses never cross members),
    generator seed (templates[m].gen_seed) and noise stream (stream_id + m); its
    g_ui of region r is scaled by g_scale[m][r] (4 receptor factors, or one per member).
    Every member starts on a 128-neuron tile: a pad region of up to 127 silent
    neurons (V_th = +inf, no noise, subblock -1) closes each member.  Subblocks are
    2 * (global region) + {0: excitatory, 1: inhibitory}.
    """
    rs, ne, sb, sc, co, cf, rm, mst, mseed, cls_rows = [0], [], [], [], [], [], [], [], [], []
    pos = 0
    rbase = 0
    for m, t in enumerate(templates):
        mst.append(pos)
        mseed.append(int(t.gen_seed))
        Rm = t.R
        first_off = len(cf)
        for r in range(Rm):
            rs.append(pos + int(t.region_start[r + 1]))
            ne.append(int(t.region_n_exc[r]))
            sb.append(rbase)
            sc.append(Rm)
            co.append(len(cf))
            cf.extend(np.asarray(t.cum[r], np.float32).tolist())
            rm.append(m)
            f = np.ones(4, np.float32)
            if g_scale is not None:
                gs = np.asarray(g_scale[m], np.float32)
                f = gs[r] if gs.ndim == 2 else gs
            for k in (0, 1):
                row = t.class_property[2 * r + k].copy()
                row[10:14] = row[10:14] * f
                row[3] = 2 * (rbase + r) + k
                cls_rows.append(row)
        pos += t.N
        pad = (-pos) % 128
        rs.append(pos + pad)
        ne.append(pad)
        sb.append(rbase)
        sc.append(Rm)
        co.append(first_off)
        rm.append(m)
        for k in (0, 1):
            row = t.class_property[0].copy()
            row[0] = 0.0            # no noise
            row[8] = np.inf         # never reaches threshold
            row[3] = -1.0           # not counted
            cls_rows.append(row)
        pos += pad
        rbase += Rm + 1
    members = dict(src_base=np.array(sb, np.int32), src_count=np.array(sc, np.int32),
                   cum_off=np.array(co, np.int64), cum_flat=np.array(cf, np.float32),
                   region_member=np.array(rm, np.int32), member_start=np.array(mst, np.int64),
                   member_seed=np.array(mseed, np.uint64))
    K = templates[0].K
    assert all(t.K == K for t in templates), "members share one in-degree"
    dt = templates[0].dt
    R = len(rs) - 1
    return NetworkSpec(name=name, region_start=np.array(rs, np.int64), region_n_exc=np.array(ne, np.int64),
                       cum=np.ones((1, 1), np.float32), K=K, class_property=np.stack(cls_rows).astype(np.float32),
                       gen_seed=int(templates[0].gen_seed), w_scale=templates[0].w_scale, dt=dt,
                       seed=templates[0].seed, stream_id=stream_id, members=members,
                       extra=dict(member_regions=[t.R for t in templates], member_sizes=[t.N for t in templates]))


def member_region_index(spec: NetworkSpec, m: int, r: int) -> int:
    """Global region index of region r of member m in an ensemble spec."""
    return int(np.nonzero(spec.members["region_member"] == m)[0][0]) + r


# Benchmark configurations (sizes and parameters of the reference's workloads).
def config_single_block() -> NetworkSpec:
    """N=2,000 (1,600 E / 400 I), K=100, dt=0.1 ms, noise p=0.01, Philox seed 0."""
    return single_block(2000, 100, name="single_block_2k")


def config_one_region(noise_rate: float = 0.01) -> NetworkSpec:
    """N=1,000,000 (80/20), K=100 (1e8 synapses)."""
    return single_block(1_000_000, 100, noise_rate=noise_rate, name=f"one_region_1M_p{noise_rate}")


def config_whole_brain(scale: float = 1.0) -> NetworkSpec:
    """90 regions, log-normal(ln 2.2e5, 0.5) sizes (~2e7 neurons), K=100 (~2e9 synapses)."""
    return whole_brain(90, 2.2e5, 0.5, 100, scale=scale, name="whole_brain_90" + ("" if scale == 1.0 else f"_x{scale}"))


def ensemble_members(n_members: int = 64, n_min: int = 50_000, n_max: int = 400_000, K: int = 100,
                     seed: int = 0, scale: float = 1.0):
    """Members of the batched-ensemble workload: neuron counts U[n_min, n_max] (times `scale`),
    one 80/20 block each with its own generator seed, and per-member g_ui factors U[0.5, 1.5]
    for the four receptors (data_assimilation/DataAssimilation.py:97 concatenates members; the
    per-member factors are cuda/python/dist_blockwrapper_pytorch.py:446-458 scalings)."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(n_min, n_max + 1, n_members)
    sizes = np.maximum(np.round(sizes * scale), 2 * K + 2).astype(np.int64)
    g_scale = rng.uniform(0.5, 1.5, (n_members, 4)).astype(np.float32)
    members = [single_block(int(n), K, gen_seed=seed * 1000 + m, name=f"member{m}") for m, n in enumerate(sizes)]
    return members, g_scale


def config_ensemble(n_members: int = 64, scale: float = 1.0, seed: int = 0) -> NetworkSpec:
    """64 members, N ~ U[5e4, 4e5] each (~1.4e7 neurons, ~1.4e9 synapses in all), K=100,
    per-member g_ui U[0.5, 1.5] x the single-block values, one BOLD region per member."""
    members, g_scale = ensemble_members(n_members, seed=seed, scale=scale)
    spec = ensemble(members, g_scale=g_scale, name=f"ensemble_{n_members}" + ("" if scale == 1.0 else f"_x{scale}"))
    spec.extra["g_scale"] = g_scale
    return spec
