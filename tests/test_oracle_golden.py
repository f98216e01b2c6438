"""The CPU oracle against the reference's own outputs (golden fixtures made by
tests/golden/make_golden.py from models/block.py and models/bold_model_pytorch.py)."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from digital_twin_brain_b200 import synthetic
from tests._helpers import GOLDEN, decay_like_reference, load_npz_blocks, schedule_steps, unpack

# Philox4x32-10 known-answer vectors published with the algorithm (Random123 kat_vectors).
KAT = [((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
       ((0xffffffff,) * 4, (0xffffffff,) * 2, (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
       ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
        (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1))]


@pytest.mark.parametrize("ctr,key,expect", KAT)
def test_philox_known_answers(ctr, key, expect):
    assert [int(x) for x in O.philox4x32_10(ctr, key)] == list(expect)
    assert [int(x) for x in O.philox4x32_10_numpy(np.array([ctr], np.uint32), key)[0]] == list(expect)


def test_noise_stream_c_matches_numpy():
    for n, step, stream in ((1, 0, 0), (1000, 7, 3), (4099, 123456789012, 5)):
        assert np.array_equal(O.noise_uniforms(99, step, n, stream), O.noise_uniforms_numpy(99, step, n, stream))


def test_noise_is_uniform():
    u = O.noise_uniforms(0, 0, 1 << 16)
    assert 0.0 <= u.min() and u.max() < 1.0
    assert abs(u.mean() - 0.5) < 0.01
    assert abs((u < 0.01).mean() - 0.01) < 0.002


def _run_oracle_schedule(prop, post, pre, kind, w, dt, seed, steps_iter, update=None, record_every=1):
    N = prop.shape[0]
    rowptr, ppre, pkind, pw = O.pull_csr(N, post, pre, kind, w)
    ob = O.OracleBlock(prop, decay_like_reference(prop, dt), rowptr, ppre, pkind, pw, dt, seed)
    act, nact, sums, means, V = [], [], [], [], []
    for k, (rate, iso) in enumerate(steps_iter):
        if update is not None and k == update[0]:
            ob.update_property(update[1], decay_like_reference(update[1], dt))
        s, m = ob.run(rate, iso)
        act.append(ob.active.astype(bool).copy())
        nact.append(ob.new_active.astype(bool).copy())
        sums.append(s)
        means.append(m)
        if (k + 1) % record_every == 0:
            V.append(ob.V.copy())
    return ob, np.stack(act), np.stack(nact), np.stack(sums), np.stack(means), np.stack(V)


def test_oracle_small_blocks_bit_exact():
    g = np.load(os.path.join(GOLDEN, "small_blocks_ref.npz"))
    prop, post, pre, kind, w = load_npz_blocks(os.path.join(GOLDEN, "small_blocks"))
    N = prop.shape[0]
    ob, act, nact, sums, means, V = _run_oracle_schedule(
        prop, post, pre, kind, w, float(g["dt"]), int(g["seed"]), schedule_steps(g["schedule"]),
        update=(int(g["update_step"]), g["new_property"]))
    assert np.array_equal(act, unpack(g["active"], N))
    assert np.array_equal(nact, unpack(g["new_active"], N))
    assert np.array_equal(V, g["V"])
    assert np.array_equal(sums, g["sums"])
    np.testing.assert_allclose(means, g["means"], rtol=2e-6)
    assert np.array_equal(ob.J, g["J_final"])
    assert np.array_equal(ob.Iui, g["I_ui_final"])
    assert np.array_equal(ob.Isyn, g["I_syn_final"])
    assert np.array_equal(ob.tlast, g["t_last_final"])
    assert np.float32(ob.t[0]) == g["t_final"]


def test_oracle_single_block_bit_exact():
    g = np.load(os.path.join(GOLDEN, "single_block_2k.npz"))
    spec = synthetic.config_single_block()
    rowptr, pre, kind, w = O.gen_network(spec.as_dict())
    post = np.repeat(np.arange(spec.N), spec.K)
    steps = int(g["steps"])
    ob, act, nact, sums, means, V = _run_oracle_schedule(
        spec.property(), post, pre.astype(np.int64), kind, w, spec.dt, spec.seed,
        ((0.01, False) for _ in range(steps)), record_every=int(g["v_every"]))
    assert np.array_equal(act, unpack(g["active"], spec.N))
    assert np.array_equal(nact, unpack(g["new_active"], spec.N))
    assert np.array_equal(V, g["V"])
    assert np.array_equal(sums, g["sums"])
    np.testing.assert_allclose(means, g["means"], rtol=2e-6)
    assert np.array_equal(ob.J, g["J_final"])
    assert np.array_equal(ob.Isyn, g["I_syn_final"])
    assert np.array_equal(ob.tlast, g["t_last_final"])


@pytest.mark.parametrize("name,dtype,rtol", [("f32", np.float32, 2e-6), ("f64", np.float64, 1e-13)])
def test_oracle_bold_against_reference(name, dtype, rtol):
    g = np.load(os.path.join(GOLDEN, "bold_ref.npz"))
    us = g[f"u_{name}"].astype(dtype)
    R = us.shape[1]
    s, q = np.zeros(R, dtype), np.zeros(R, dtype)
    v, f = np.ones(R, dtype), np.ones(R, dtype)
    params = dict(epsilon=200, tao_s=0.8, tao_f=0.4, tao_0=1, alpha=0.2, E_0=0.8, V_0=0.02)
    outs = np.stack([O.bold_step(us[k].copy(), s, q, v, f, params, float(g["delta_t"])) for k in range(len(us))])
    np.testing.assert_allclose(outs, g[f"bold_{name}"], rtol=rtol, atol=0)
    for fld, arr in (("s", s), ("q", q), ("v", v), ("f_in", f)):
        np.testing.assert_allclose(arr, g[f"{fld}_{name}"], rtol=rtol, atol=1e-30)


def test_generator_rows_are_deterministic_and_valid():
    spec = synthetic.whole_brain(R=5, mean_size=400, sigma=0.5, K=20, gen_seed=3)
    pre_a, kind_a, w_a = O.gen_rows(spec.as_dict(), 0, spec.N)
    pre_b, kind_b, w_b = O.gen_rows(spec.as_dict(), 100, 200)
    K = spec.K
    assert np.array_equal(pre_a[100 * K:200 * K], pre_b) and np.array_equal(w_a[100 * K:200 * K], w_b)
    rows = pre_a.reshape(spec.N, K).astype(np.int64)
    assert (np.diff(rows, axis=1) > 0).all()                      # sorted, distinct
    assert not (rows == np.arange(spec.N)[:, None]).any()         # no self connection
    region = np.searchsorted(spec.region_start, rows, side="right") - 1
    exc = (rows - spec.region_start[region]) < spec.region_n_exc[region]
    assert np.array_equal(kind_a.reshape(spec.N, K), np.where(exc, 0, 2))
    own = region == (np.searchsorted(spec.region_start, np.arange(spec.N), side="right") - 1)[:, None]
    assert abs(own.mean() - 0.8) < 0.03                            # 80 % intra-region
    assert 0.0 <= w_a.min() and w_a.max() < 1.0


def test_ensemble_members_equal_standalone_networks():
    """Members of a concatenated ensemble keep their own connectivity (member-local generator counters)."""
    t = [synthetic.single_block(500, 20, gen_seed=11, name="m0"),
         synthetic.whole_brain(R=3, mean_size=300, sigma=0.3, K=20, gen_seed=12, name="m1"),
         synthetic.single_block(300, 20, gen_seed=13, name="m2")]
    e = synthetic.ensemble(t, g_scale=np.array([[1, 1, 1, 1], [1.2, 0.8, 1, 1], [0.5, 1, 1.5, 1]], np.float32))
    assert (e.members["member_start"] % 128 == 0).all()
    pe, ke, we = O.gen_rows(e.as_dict(), 0, e.N)
    K = e.K
    for m, tm in enumerate(t):
        ps, ks, ws = O.gen_rows(tm.as_dict(), 0, tm.N)
        ms = int(e.members["member_start"][m])
        seg = slice(ms * K, (ms + tm.N) * K)
        assert np.array_equal(pe[seg].astype(np.int64) - ms, ps.astype(np.int64))
        assert np.array_equal(ke[seg], ks) and np.array_equal(we[seg], ws)


def test_oracle_input_neurons_vs_reference():
    """models/block.py with src (input neurons replaying a raster), run by the reference itself."""
    g = np.load(os.path.join(GOLDEN, "src_block_ref.npz"))
    prop, src = g["prop"], g["src"]
    N = prop.shape[0]
    n_src = src.shape[0]
    rp, pre, kind, w = O.pull_csr(N, g["post"], g["pre"], g["kind"], g["w"])
    ob = O.OracleBlock(prop, decay_like_reference(prop, float(g["dt"])), rp, pre, kind, w, float(g["dt"]),
                       int(g["seed"]))
    act = unpack(g["active"], N)
    for k in range(int(g["steps"])):
        fa = np.full(N, 2, np.uint8)
        fa[:n_src] = src[:, k]
        s, m = ob.run(0.01, forced_active=fa)
        assert np.array_equal(ob.active.astype(bool), act[k]), k
        assert np.array_equal(ob.V, g["V"][k]), k
        assert np.array_equal(s, g["sums"][k])
    assert np.array_equal(ob.J, g["J_final"])
    assert np.array_equal(ob.Isyn, g["I_syn_final"])
    assert np.array_equal(ob.tlast, g["t_last_final"])
