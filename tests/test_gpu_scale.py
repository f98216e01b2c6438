"""Parity at the sizes the benchmark runs.

* One region of 1e6 neurons and 1e8 synapses (K = 100, p = 0.01): DTB_MODE_PULL equal
  to the oracle's restatement of models/block.py bit for bit for 150 steps (100 past
  the 50-step refractory window every neuron starts in); the push step (float2
  atomics with the whole-brain autotuned launch shape and staged update, and the
  binned push) under teacher forcing within 1e-5 of the oracle.
* The whole-brain network (90 regions, 2.34e7 neurons, 2.34e9 synapses): the
  device generator's pull rows sampled everywhere (rows past entry 2^31 included)
  against the oracle's generator; the push CSR's row lengths against the
  out-degrees counted over every pull entry, sampled push rows against the pull
  rows they came from; two teacher-forced push steps of sampled neurons against a
  float32 restatement of models/block.py:68-114 fed the same state and spikes.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from digital_twin_brain_b200 import Network, synthetic
from digital_twin_brain_b200._lib import (FIELD_ACTIVE, FIELD_J, FIELD_NEW_ACTIVE, FIELD_T, FIELD_T_LAST, FIELD_V,
                                          TUNE_PUSH_METHOD, TUNE_SCATTER_WORDS, TUNE_STEP_VARIANT)
from tests._helpers import decay_like_reference

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

KIND = np.uint32(0x80000000)
ATOMIC, BINNED = 1, 2


def _class_decay(spec):
    """exp(-dt/tau) per class as models/block.py:71 evaluates it (elementwise, so per class = per neuron)."""
    return np.ascontiguousarray(decay_like_reference(spec.class_property, spec.dt).T)


# ---------------------------------------------------------------- one region, 1e6 neurons

@pytest.fixture(scope="module")
def one_region():
    spec = synthetic.config_one_region(0.01)
    rowptr, pre, kind, w = O.gen_network(spec.as_dict())
    return spec, (rowptr, pre, kind, w)


def _oracle(spec, csr):
    prop = spec.property()
    return O.OracleBlock(prop, decay_like_reference(prop, spec.dt), *csr, spec.dt, spec.seed)


def test_one_region_pull_bit_exact_vs_oracle(one_region):
    spec, csr = one_region
    net = Network.from_spec(spec, device=0, class_decay=_class_decay(spec))
    ob = _oracle(spec, csr)
    steps = 150
    s, m, na = net.run(steps, noise_rate=0.01, mode="pull")
    for k in range(steps):
        so, mo = ob.run(0.01)
        assert np.array_equal(s[k], so), f"spike counts differ at step {k}"
        np.testing.assert_allclose(m[k], mo, rtol=2e-6)
        assert na[k] == int(ob.new_active.sum())
    assert s[60:].sum() > 1000                      # past the refractory window neurons fire
    assert np.array_equal(net.get(FIELD_V), ob.V)
    assert np.array_equal(net.get(FIELD_J), ob.J)
    assert np.array_equal(net.get(FIELD_T_LAST), ob.tlast)
    assert np.array_equal(net.get(FIELD_ACTIVE).astype(bool), ob.active.astype(bool))


@pytest.mark.parametrize("method", ["atomic_autotuned_shape", "binned"])
def test_one_region_push_teacher_forced_vs_oracle(one_region, method):
    spec, csr = one_region
    net = Network.from_spec(spec, device=0, class_decay=_class_decay(spec))
    if method == "binned":
        net.set_tuning(TUNE_PUSH_METHOD, BINNED)
    else:   # the whole-brain bench's autotuned atomic launch: 4 words per warp, staged update (3 CTAs/SM)
        net.set_tuning(TUNE_PUSH_METHOD, ATOMIC)
        net.set_tuning(TUNE_SCATTER_WORDS, 4)
        net.set_tuning(TUNE_STEP_VARIANT, 3)
    ob = _oracle(spec, csr)
    for k in range(110):
        so, _ = ob.run(0.01)
        s, _ = net.step_forced(ob.active, ob.new_active, noise_rate=0.01, mode="push")
        assert np.array_equal(s, so)
        if k in (59, 109):
            np.testing.assert_allclose(net.get(FIELD_V), ob.V, rtol=1e-5, atol=1e-5)
            np.testing.assert_allclose(net.get(FIELD_J), ob.J, rtol=1e-5, atol=1e-6)
            assert np.array_equal(net.get(FIELD_T_LAST), ob.tlast)


# ---------------------------------------------------------------- whole brain, 2.34e9 synapses

@pytest.fixture(scope="module")
def whole_brain():
    spec = synthetic.config_whole_brain()
    net = Network.from_spec(spec, device=0, class_decay=_class_decay(spec))
    yield spec, net
    del net
    torch.cuda.empty_cache()


def _sample_rows(spec, n, rng):
    N, K = spec.N, spec.K
    past = (2 ** 31) // K + 1                       # first row whose entries lie past entry 2^31
    picks = [0, 1, N - 1, N - 2, past - 1, past, past + 1]
    for r in range(spec.R):                         # first and last neuron of every region
        picks += [int(spec.region_start[r]), int(spec.region_start[r + 1]) - 1]
    picks += list(rng.integers(0, N, n))
    picks += list(rng.integers(past, N, n // 4))
    return np.unique(np.asarray(picks, np.int64))


def test_whole_brain_generator_rows_vs_oracle(whole_brain):
    spec, net = whole_brain
    N, K = spec.N, spec.K
    assert net.S == N * K and net.S > 2 ** 31
    rp = net.get_csr_rowptr("pull")
    assert np.array_equal(rp, np.arange(N + 1, dtype=np.int64) * K)
    d = spec.as_dict()
    for r in _sample_rows(spec, 400, np.random.default_rng(1)):
        ix, w = net.get_csr_entries("pull", int(r) * K, K)
        pre, kind, ow = O.gen_rows(d, int(r), int(r) + 1)
        assert np.array_equal(ix, pre | np.where(kind == 2, KIND, np.uint32(0))), f"row {r}"
        assert np.array_equal(w, ow), f"row {r}"


def test_whole_brain_push_csr_vs_pull(whole_brain):
    spec, net = whole_brain
    N, K, S = spec.N, spec.K, net.S
    qrp = net.get_csr_rowptr("push")
    assert qrp[0] == 0 and qrp[-1] == S and np.all(np.diff(qrp) >= 0)
    # out-degree of every neuron counted over all 2.34e9 pull entries, on the device
    dev = torch.device("cuda", 0)
    counts = torch.zeros(N, dtype=torch.int64, device=dev)
    chunk = 1 << 28
    for e0 in range(0, S, chunk):
        ix, _ = net.get_csr_entries("pull", e0, min(chunk, S - e0), device=True, weights=False)
        counts += torch.bincount((ix & 0x7FFFFFFF).to(torch.int64), minlength=N)
        del ix
    assert np.array_equal(np.diff(qrp), counts.cpu().numpy())
    # sampled push rows: every entry is the pull entry (post, pre, kind, w) it came from; posts ascend
    d = spec.as_dict()
    for i in _sample_rows(spec, 150, np.random.default_rng(2)):
        e0, e1 = int(qrp[i]), int(qrp[i + 1])
        if e1 == e0:
            continue
        qix, qw = net.get_csr_entries("push", e0, e1 - e0)
        post = (qix & 0x7FFFFFFF).astype(np.int64)
        assert np.all(np.diff(post) > 0), f"push row {i} not ascending"
        for p, kbit, ww in zip(post, qix >> 31, qw):
            pre, kind, ow = O.gen_rows(d, int(p), int(p) + 1)
            hit = np.nonzero(pre == i)[0]
            assert len(hit) == 1, f"push entry ({i} -> {p}) has no pull entry"
            assert (kind[hit[0]] == 2) == bool(kbit) and np.array_equal(ow[hit[0]], ww)


def _restated_step(spec, dec, cls, V, J, tl, t_prev, act, new, rows_pre, rows_kind, rows_w):
    """models/block.py:68-114 for the sampled neurons (float32, the reference's operation order)."""
    f = np.float32
    P = spec.class_property[cls]
    g, Vu = P[:, 10:14].T.astype(f), P[:, 14:18].T.astype(f)
    i_ui = (g * (Vu - V[None, :])) * J
    isyn = ((i_ui[0] + i_ui[1]) + i_ui[2]) + i_ui[3]
    t = f(t_prev + f(spec.dt))
    rcdt = (f(1.0) / P[:, 4].astype(f)) * f(spec.dt)
    main = (-P[:, 6].astype(f)) * (V - P[:, 7].astype(f))
    vn = V + rcdt * ((main + isyn) + P[:, 2].astype(f))
    notsat = t >= tl + P[:, 5].astype(f)
    vs = np.where(notsat, vn, P[:, 9].astype(f))
    Vnew = np.minimum(vs, P[:, 8].astype(f))
    tlnew = np.where(act, t, tl)
    fired = new[rows_pre]                                  # [n, K]
    inh = rows_kind == 2
    add = np.zeros((4, len(V)), np.float64)
    for c, sel in ((0, ~inh), (2, inh)):
        m = fired & sel
        add[c] = (rows_w[..., 0] * m).sum(1)
        add[c + 1] = (rows_w[..., 1] * m).sum(1)
    Jnew = J * dec[cls].T + add.astype(f)
    return Vnew.astype(f), Jnew, tlnew


@pytest.mark.parametrize("method", [BINNED, ATOMIC], ids=["binned", "atomic"])
def test_whole_brain_teacher_forced_push_sampled_vs_restatement(whole_brain, method):
    spec, net = whole_brain
    N, K = spec.N, spec.K
    net.set_tuning(TUNE_PUSH_METHOD, method)
    net.run(60, noise_rate=0.01, mode="push")           # leave the refractory window
    rng = np.random.default_rng(3 + method)
    sample = _sample_rows(spec, 3000, rng)
    d = spec.as_dict()
    rows = [O.gen_rows(d, int(n), int(n) + 1) for n in sample]
    rows_pre = np.stack([r[0] for r in rows]).astype(np.int64)
    rows_kind = np.stack([r[1] for r in rows])
    rows_w = np.stack([r[2] for r in rows])
    cls = spec.neuron_class()[sample]
    dec = _class_decay(spec)
    for step in range(2):
        V, J, tl, t = net.get(FIELD_V), net.get(FIELD_J), net.get(FIELD_T_LAST), net.get(FIELD_T)
        act = rng.random(N) < 0.005
        new = act | (rng.random(N) < 0.005)
        net.step_forced(act.astype(np.uint8), new.astype(np.uint8), noise_rate=0.01, mode="push")
        Ve, Je, tle = _restated_step(spec, dec, cls, V[sample], J[:, sample], tl[sample], np.float32(t),
                                     act[sample], new, rows_pre, rows_kind, rows_w)
        assert np.array_equal(net.get(FIELD_V)[sample], Ve), f"V differs at forced step {step}"
        assert np.array_equal(net.get(FIELD_T_LAST)[sample], tle)
        np.testing.assert_allclose(net.get(FIELD_J)[:, sample], Je, rtol=1e-5, atol=1e-6)
        assert np.array_equal(net.get(FIELD_NEW_ACTIVE).astype(bool), new)
