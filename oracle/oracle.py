"""CPU oracle — test infrastructure only.

Python side of the oracle: a ctypes wrapper around ``liboracle.so``
(``oracle/oracle.c``) plus numpy restatements of the parts of the reference
that are pure data handling.  Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU baseline / reference arm import this module; the product
(``digital_twin_brain_b200``) never does.

Reference behaviour restated here:

* ``generation/read_block.py:64-90`` — an npz block becomes COO entries
  ``(channel, post, pre)`` duplicated for ``channel+1``; ``torch.sparse.mm``
  then accumulates each postsynaptic row in nnz (file) order, so the pull CSR
  is a *stable* sort of the entries by postsynaptic index (:func:`pull_csr`).
* ``cuda/src/configuration.cpp:575-828`` — the native push CSR is a stable
  sort of the same entries by presynaptic key (:func:`push_csr`).
* ``models/block.py:144-150`` — per-subblock spike sums and mean V
  (:func:`subblock_stats`).
* ``models/block.py:30-60`` — initial state (:class:`OracleBlock`).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

u32 = ctypes.c_uint32
i64 = ctypes.c_int64
u64 = ctypes.c_uint64
f32 = ctypes.c_float
f64 = ctypes.c_double
vp = ctypes.c_void_p


def build() -> str:
    """Compile ``liboracle.so`` with the committed Makefile (gcc, OpenMP)."""
    path = os.path.join(_HERE, "liboracle.so")
    src = os.path.join(_HERE, "oracle.c")
    if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE])
    return path


def lib():
    global _LIB
    if _LIB is None:
        L = ctypes.CDLL(build())
        L.oracle_philox4x32_10.argtypes = [vp, vp, vp]
        L.oracle_noise_uniforms.argtypes = [u64, u32, u64, i64, vp]
        L.oracle_block_step.argtypes = [i64] + [vp] * 10 + [vp] * 4 + [vp] * 5 + [f32, f32, vp, u64, u32, u64,
                                                                              ctypes.c_int, vp, vp, vp, vp, vp,
                                                                              ctypes.c_int]
        L.oracle_block_step.restype = ctypes.c_int
        L.oracle_bold_step_f32.argtypes = [i64] + [vp] * 6 + [f64] * 8
        L.oracle_bold_step_f64.argtypes = [i64] + [vp] * 6 + [f64] * 8
        L.oracle_gen_rows.argtypes = [ctypes.c_int] + [vp] * 9 + [ctypes.c_int, f32, i64, i64, vp, vp, vp]
        L.oracle_gamma.argtypes = [i64, vp, f64, f64, ctypes.c_int, u32, u64, vp]
        L.oracle_gamma.restype = None
        L.oracle_gen_rows.restype = ctypes.c_int
        _LIB = L
    return _LIB


def _p(a: np.ndarray):
    return a.ctypes.data_as(vp) if a is not None else None


# ----------------------------------------------------------------- Philox

def philox4x32_10(ctr, key):
    c = np.ascontiguousarray(np.asarray(ctr, dtype=np.uint32))
    k = np.ascontiguousarray(np.asarray(key, dtype=np.uint32))
    o = np.zeros(4, np.uint32)
    lib().oracle_philox4x32_10(_p(c), _p(k), _p(o))
    return o


def philox4x32_10_numpy(ctr: np.ndarray, key) -> np.ndarray:
    """Vectorised numpy Philox4x32-10 (Salmon et al., SC'11); ctr is [n,4] uint32."""
    c = [ctr[:, j].astype(np.uint64) for j in range(4)]
    k0 = np.uint64(int(key[0]) & 0xFFFFFFFF)
    k1 = np.uint64(int(key[1]) & 0xFFFFFFFF)
    M = np.uint64(0xFFFFFFFF)
    for r in range(10):
        if r:
            k0 = (k0 + np.uint64(0x9E3779B9)) & M
            k1 = (k1 + np.uint64(0xBB67AE85)) & M
        p0 = np.uint64(0xD2511F53) * c[0]
        p1 = np.uint64(0xCD9E8D57) * c[2]
        hi0, lo0 = p0 >> np.uint64(32), p0 & M
        hi1, lo1 = p1 >> np.uint64(32), p1 & M
        c = [hi1 ^ c[1] ^ k0, lo1, hi0 ^ c[3] ^ k1, lo0]
    return np.stack([x.astype(np.uint32) for x in c], axis=1)


def noise_uniforms(seed: int, step: int, n: int, stream: int = 0) -> np.ndarray:
    out = np.empty(n, np.float32)
    lib().oracle_noise_uniforms(seed, stream, step, n, _p(out))
    return out


def noise_uniforms_numpy(seed: int, step: int, n: int, stream: int = 0) -> np.ndarray:
    """Same stream as :func:`noise_uniforms`, computed with numpy only."""
    groups = (n + 127) // 128
    q = np.arange(groups * 32, dtype=np.uint64)
    ctr = np.stack([q.astype(np.uint32), np.full_like(q, stream).astype(np.uint32),
                    np.full_like(q, step & 0xFFFFFFFF).astype(np.uint32),
                    np.full_like(q, step >> 32).astype(np.uint32)], axis=1)
    o = philox4x32_10_numpy(ctr, (seed & 0xFFFFFFFF, seed >> 32))  # [groups*32, 4]
    u = (o >> np.uint32(8)).astype(np.float32) * np.float32(1.0 / 16777216.0)
    # neuron n = g*128 + w*32 + lane  <->  row g*32+lane, word w
    u = u.reshape(groups, 32, 4).transpose(0, 2, 1).reshape(-1)
    return u[:n].copy()


# ------------------------------------------------------------ CSR layouts

def coo_from_npz_arrays(output_neuron_idx, input_block_idx, input_neuron_idx, input_channel_offset, weight,
                        block_index: int, bases: np.ndarray):
    """generation/read_block.py:64-74 — global (post, pre, kind, w[E,2]) in file order."""
    post = output_neuron_idx.astype(np.int64) + int(bases[block_index])
    pre = (bases[(input_block_idx.astype(np.int64) + block_index)] + input_neuron_idx.astype(np.int64))
    return post, pre.astype(np.int64), input_channel_offset.astype(np.uint8), weight.reshape(-1, 2).astype(np.float32)


def pull_csr(N: int, post, pre, kind, w):
    """Stable sort by postsynaptic index: sparse.mm accumulation order per row."""
    order = np.argsort(post, kind="stable")
    counts = np.bincount(post, minlength=N)
    rowptr = np.zeros(N + 1, np.int64)
    np.cumsum(counts, out=rowptr[1:])
    return rowptr, pre[order].astype(np.uint32), kind[order].astype(np.uint8), np.ascontiguousarray(w[order])


def push_csr(N: int, post, pre, kind, w):
    """Stable sort by presynaptic index (configuration.cpp:575-828 key order)."""
    order = np.argsort(pre, kind="stable")
    counts = np.bincount(pre, minlength=N)
    rowptr = np.zeros(N + 1, np.int64)
    np.cumsum(counts, out=rowptr[1:])
    return rowptr, post[order].astype(np.uint32), kind[order].astype(np.uint8), np.ascontiguousarray(w[order])


def subblock_stats(V: np.ndarray, active: np.ndarray, sub_idx: np.ndarray):
    """models/block.py:144-150 (mean V per subblock, spike sum per subblock)."""
    n_sub = int(sub_idx.max()) + 1 if sub_idx.size else 0
    sums = np.zeros(n_sub, np.float32)
    means = np.zeros(n_sub, np.float32)
    for i in range(n_sub):
        m = sub_idx == i
        sums[i] = np.float32(active[m].sum())
        means[i] = np.float32(V[m].astype(np.float64).mean()) if m.any() else np.float32(np.nan)
    return sums, means


# -------------------------------------------------------------- generator

def general_tables(spec: dict):
    """Source-region tables of a network spec (single network: every region draws from all R
    regions through its row of cum[R][R]; ensembles pass the tables explicitly)."""
    rs = np.ascontiguousarray(spec["region_start"], dtype=np.int64)
    R = len(rs) - 1
    if spec.get("src_count") is not None:
        t = dict(src_base=spec["src_base"], src_count=spec["src_count"], cum_off=spec["cum_off"],
                 cum_flat=spec["cum_flat"], region_member=spec["region_member"],
                 member_start=spec["member_start"], member_seed=spec["member_seed"])
    else:
        t = dict(src_base=np.zeros(R, np.int32), src_count=np.full(R, R, np.int32),
                 cum_off=np.arange(R, dtype=np.int64) * R, cum_flat=np.asarray(spec["cum"], np.float32).reshape(-1),
                 region_member=np.zeros(R, np.int32), member_start=np.zeros(1, np.int64),
                 member_seed=np.array([int(spec["gen_seed"])], np.uint64))
    dt = dict(src_base=np.int32, src_count=np.int32, cum_off=np.int64, cum_flat=np.float32, region_member=np.int32,
              member_start=np.int64, member_seed=np.uint64)
    return {k: np.ascontiguousarray(v, dtype=dt[k]) for k, v in t.items()}


def gen_rows(spec: dict, row_begin: int, row_end: int):
    """Rows [row_begin,row_end) of the counter-based synthetic network (oracle.c)."""
    K = int(spec["K"])
    n = row_end - row_begin
    pre = np.zeros(n * K, np.uint32)
    kind = np.zeros(n * K, np.uint8)
    w = np.zeros(n * K * 2, np.float32)
    rs = np.ascontiguousarray(spec["region_start"], dtype=np.int64)
    ne = np.ascontiguousarray(spec["region_n_exc"], dtype=np.int64)
    t = general_tables(spec)
    bad = lib().oracle_gen_rows(len(rs) - 1, _p(rs), _p(ne), _p(t["src_base"]), _p(t["src_count"]), _p(t["cum_off"]),
                                _p(t["cum_flat"]), _p(t["region_member"]), _p(t["member_start"]),
                                _p(t["member_seed"]), K, float(spec.get("w_scale", 1.0)), row_begin, row_end,
                                _p(pre), _p(kind), _p(w))
    if bad:
        raise RuntimeError(f"generator could not draw {K} distinct sources for {bad} rows")
    return pre, kind, w.reshape(-1, 2)


def gen_network(spec: dict):
    """Whole synthetic network as a pull CSR (rows sorted by presynaptic index)."""
    N = int(spec["region_start"][-1])
    K = int(spec["K"])
    pre, kind, w = gen_rows(spec, 0, N)
    rowptr = np.arange(N + 1, dtype=np.int64) * K
    return rowptr, pre, kind, w


# ------------------------------------------------------------------ block

@dataclass
class Params:
    Iext: np.ndarray
    C: np.ndarray
    Tref: np.ndarray
    gL: np.ndarray
    VL: np.ndarray
    Vth: np.ndarray
    Vreset: np.ndarray
    g: np.ndarray       # [4,N]
    Vu: np.ndarray      # [4,N]
    decay: np.ndarray   # [4,N]
    noise: np.ndarray   # [N] property column 0
    sub_idx: np.ndarray

    @staticmethod
    def from_property(prop: np.ndarray, decay: np.ndarray):
        """block.update_property column split (models/block.py:156-169)."""
        p = np.ascontiguousarray(prop, dtype=np.float32)
        c = lambda j: np.ascontiguousarray(p[:, j])
        return Params(Iext=c(2), C=c(4), Tref=c(5), gL=c(6), VL=c(7), Vth=c(8), Vreset=c(9),
                      g=np.ascontiguousarray(p[:, 10:14].T), Vu=np.ascontiguousarray(p[:, 14:18].T),
                      decay=np.ascontiguousarray(decay, dtype=np.float32), noise=c(0), sub_idx=c(3))


class OracleBlock:
    """Stateful wrapper: block.__init__ (models/block.py:53-60) + run (:116-150)."""

    def __init__(self, prop: np.ndarray, decay: np.ndarray, rowptr, pre, kind, w, dt: float, seed: int,
                 stream: int = 0, nthreads: int = 0):
        self.P = Params.from_property(prop, decay)
        self.N = prop.shape[0]
        self.rowptr = np.ascontiguousarray(rowptr, np.int64)
        self.pre = np.ascontiguousarray(pre, np.uint32)
        self.kind = np.ascontiguousarray(kind, np.uint8)
        self.w = np.ascontiguousarray(w, np.float32).reshape(-1)
        self.dt = float(dt)
        self.seed = int(seed)
        self.stream = int(stream)
        self.nthreads = int(nthreads)
        self.V = (np.ones(self.N, np.float32) * ((self.P.Vth + self.P.Vreset) / np.float32(2))).astype(np.float32)
        self.J = np.zeros((4, self.N), np.float32)
        self.tlast = np.zeros(self.N, np.float32)
        self.Isyn = np.zeros(self.N, np.float32)
        self.Iui = np.zeros((4, self.N), np.float32)
        self.t = np.zeros(1, np.float32)
        self.step_index = 0
        self.active = np.zeros(self.N, np.uint8)
        self.new_active = np.zeros(self.N, np.uint8)

    def update_property(self, prop: np.ndarray, decay: np.ndarray):
        """models/block.py:152-170: new parameters; the stored I_syn stays until the next step."""
        self.P = Params.from_property(prop, decay)

    def run(self, noise_rate: float = 0.01, isolated: bool = False, forced_active=None, forced_new_active=None):
        P = self.P
        fa = None if forced_active is None else np.ascontiguousarray(forced_active, np.uint8)
        fn = None if forced_new_active is None else np.ascontiguousarray(forced_new_active, np.uint8)
        rc = lib().oracle_block_step(
            self.N, _p(P.Iext), _p(P.C), _p(P.Tref), _p(P.gL), _p(P.VL), _p(P.Vth), _p(P.Vreset),
            _p(P.g), _p(P.Vu), _p(P.decay), _p(self.rowptr), _p(self.pre), _p(self.kind), _p(self.w),
            _p(self.V), _p(self.J), _p(self.tlast), _p(self.Isyn), _p(self.t), self.dt,
            float(noise_rate) if noise_rate is not None else -1.0, _p(P.noise),
            self.seed, self.stream, self.step_index, int(bool(isolated)), _p(fa), _p(fn),
            _p(self.active), _p(self.new_active), _p(self.Iui), self.nthreads)
        if rc != 0:
            raise MemoryError("oracle_block_step failed")
        self.step_index += 1
        return subblock_stats(self.V, self.active, P.sub_idx)


def gamma(neurons, alpha: float, beta: float, receptor: int, call: int, seed: int) -> np.ndarray:
    """Per-neuron Gamma(alpha, 1) / beta draws of the product's gamma-distributed g_ui (float32)."""
    idx = np.ascontiguousarray(neurons, np.int64)
    out = np.empty(len(idx), np.float32)
    lib().oracle_gamma(len(idx), _p(idx), float(alpha), float(beta), int(receptor), int(call), int(seed), _p(out))
    return out


def bold_step(u, s, q, v, f, params: dict, delta_t: float):
    """BOLD.run (models/bold_model_pytorch.py:43-78) on numpy arrays (float32 or float64)."""
    fn = lib().oracle_bold_step_f64 if u.dtype == np.float64 else lib().oracle_bold_step_f32
    out = np.empty_like(u)
    fn(u.size, _p(u), _p(s), _p(q), _p(v), _p(f), _p(out), float(params["epsilon"]), float(params["tao_s"]),
       float(params["tao_f"]), float(params["tao_0"]), float(params["alpha"]), float(params["E_0"]),
       float(params["V_0"]), float(delta_t))
    return out
