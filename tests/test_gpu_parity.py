"""CUDA path (libdtb through its C ABI and the drop-in classes) against the
reference's golden outputs and the CPU oracle."""
import os

import numpy as np
import pytest
import torch

from oracle import oracle as O
from digital_twin_brain_b200 import Network, synthetic
from digital_twin_brain_b200._lib import (FIELD_ACTIVE, FIELD_I_SYN, FIELD_I_UI, FIELD_J, FIELD_NEW_ACTIVE,
                                          FIELD_T, FIELD_T_LAST, FIELD_V)
from tests._helpers import GOLDEN, decay_like_reference, load_npz_blocks, schedule_steps, unpack

pytestmark = pytest.mark.gpu

KIND = np.uint32(0x80000000)


def class_decay_like_reference(spec):
    """Per-class exp(-dt/tau), taken from the reference-style evaluation over all neurons."""
    prop = spec.property()
    d = decay_like_reference(prop, spec.dt).T  # [N,4]
    cls = spec.neuron_class()
    out = np.zeros((2 * spec.R, 4), np.float32)
    for c in range(2 * spec.R):
        rows = d[cls == c]
        if len(rows):
            assert (rows == rows[0]).all()
            out[c] = rows[0]
        else:
            out[c] = decay_like_reference(spec.class_property[c:c + 1], spec.dt).T[0]
    return out


def reference_sparse_w(post, pre, kind, w, N):
    """The [4,N,N] torch sparse tensor generation/read_block.py:68-90 builds (uncoalesced, file order)."""
    idx = np.stack([kind.astype(np.int64), post.astype(np.int64), pre.astype(np.int64)])
    idx = np.stack([idx, idx], axis=-1)
    idx[0, :, 1] += 1
    idx = idx.reshape(3, -1)
    return torch.sparse_coo_tensor(torch.from_numpy(idx), torch.from_numpy(w.reshape(-1).copy()), (4, N, N))


# ---------------------------------------------------------------- generator / CSR

@pytest.mark.parametrize("spec", [synthetic.config_single_block(),
                                  synthetic.whole_brain(R=6, mean_size=600, sigma=0.5, K=40, gen_seed=5)],
                         ids=["single_block", "whole_brain_small"])
def test_generator_and_csr_bit_exact(spec):
    net = Network.from_spec(spec, device=0, build_push=True)
    rp, ix, w = net.get_csr("pull")
    orp, opre, okind, ow = O.gen_network(spec.as_dict())
    assert np.array_equal(rp, orp)
    assert np.array_equal(ix, opre | np.where(okind == 2, KIND, np.uint32(0)))
    assert np.array_equal(w, ow)
    # push CSR: transposition, rows sorted by postsynaptic index
    post = np.repeat(np.arange(spec.N), spec.K)
    qrp, qpost, qkind, qw = O.push_csr(spec.N, post, opre.astype(np.int64), okind, ow)
    prp, pix, pw = net.get_csr("push")
    assert np.array_equal(prp, qrp)
    assert np.array_equal(pix, qpost | np.where(qkind == 2, KIND, np.uint32(0)))
    assert np.array_equal(pw, qw)


def test_npz_loader_csr_matches_reference_order():
    d = os.path.join(GOLDEN, "small_blocks")
    prop, post, pre, kind, w = load_npz_blocks(d)
    N = prop.shape[0]
    net = Network.from_npz(d, dt=0.1, seed=11, device=0, build_push=True)
    assert net.N == N and net.S == len(post)
    for which, builder in (("pull", O.pull_csr), ("push", O.push_csr)):
        rp, ix, ww = net.get_csr(which)
        orp, oidx, okind, ow = builder(N, post, pre, kind, w)
        assert np.array_equal(rp, orp)
        assert np.array_equal(ix, oidx | np.where(okind == 2, KIND, np.uint32(0)))
        assert np.array_equal(ww, ow)


# ---------------------------------------------------------------- block step vs reference

def test_single_block_pull_bit_exact_vs_reference():
    g = np.load(os.path.join(GOLDEN, "single_block_2k.npz"))
    spec = synthetic.config_single_block()
    net = Network.from_spec(spec, device=0, build_push=True, class_decay=class_decay_like_reference(spec))
    every = int(g["v_every"])
    steps = int(g["steps"])
    act_ref = unpack(g["active"], spec.N)
    nact_ref = unpack(g["new_active"], spec.N)
    for c in range(steps // every):
        s, m, na = net.run(every, noise_rate=0.01, mode="pull")
        k = (c + 1) * every - 1
        assert np.array_equal(s, g["sums"][c * every:(c + 1) * every])
        np.testing.assert_allclose(m, g["means"][c * every:(c + 1) * every], rtol=2e-6)
        assert np.array_equal(na, nact_ref[c * every:(c + 1) * every].sum(1))
        assert np.array_equal(net.get(FIELD_V), g["V"][c]), f"V differs after step {k}"
        assert np.array_equal(net.get(FIELD_ACTIVE).astype(bool), act_ref[k])
        assert np.array_equal(net.get(FIELD_NEW_ACTIVE).astype(bool), nact_ref[k])
    assert np.array_equal(net.get(FIELD_J), g["J_final"])
    assert np.array_equal(net.get(FIELD_I_SYN), g["I_syn_final"])
    assert np.array_equal(net.get(FIELD_T_LAST), g["t_last_final"])
    assert np.float32(net.get(FIELD_T)) == g["t_final"]


def test_small_blocks_drop_in_bit_exact_vs_reference():
    """The drop-in block class, fed exactly what generation/read_block.py gives the reference."""
    from digital_twin_brain_b200.models.block import block
    g = np.load(os.path.join(GOLDEN, "small_blocks_ref.npz"))
    prop, post, pre, kind, w = load_npz_blocks(os.path.join(GOLDEN, "small_blocks"))
    N = prop.shape[0]
    W = reference_sparse_w(post, pre, kind, w, N)
    b = block(torch.from_numpy(prop), W, delta_t=float(g["dt"]), seed=int(g["seed"]), device=0)
    act_ref = unpack(g["active"], N)
    for k, (rate, iso) in enumerate(schedule_steps(g["schedule"])):
        if k == int(g["update_step"]):
            b.update_property(torch.from_numpy(g["new_property"]))
        s, m = b.run(noise_rate=rate, isolated=iso)
        assert np.array_equal(s.numpy(), g["sums"][k])
        np.testing.assert_allclose(m.numpy(), g["means"][k], rtol=2e-6)
        assert np.array_equal(b.active.numpy(), act_ref[k]), f"spikes differ at step {k}"
        assert np.array_equal(b.V_i.numpy(), g["V"][k]), f"V differs at step {k}"
    assert np.array_equal(b.J_ui.numpy(), g["J_final"])
    assert np.array_equal(b.I_ui.numpy(), g["I_ui_final"])
    assert np.array_equal(b.I_syn.numpy(), g["I_syn_final"])
    assert np.array_equal(b.t_ik_last.numpy(), g["t_last_final"])
    assert np.float32(b.t.item()) == g["t_final"]


@pytest.mark.parametrize("push_method", [1, 2], ids=["atomic", "binned"])
def test_push_teacher_forced_within_tolerance(push_method):
    """Push scatter (float atomics, any order; or binned) under teacher forcing: V and J within 1e-5 relative."""
    from digital_twin_brain_b200._lib import TUNE_PUSH_METHOD
    g = np.load(os.path.join(GOLDEN, "single_block_2k.npz"))
    spec = synthetic.config_single_block()
    net = Network.from_spec(spec, device=0, build_push=True, class_decay=class_decay_like_reference(spec))
    net.set_tuning(TUNE_PUSH_METHOD, push_method)
    act_ref = unpack(g["active"], spec.N)
    nact_ref = unpack(g["new_active"], spec.N)
    every = int(g["v_every"])
    for k in range(int(g["steps"])):
        s, _ = net.step_forced(act_ref[k], nact_ref[k], noise_rate=0.01, mode="push")
        assert np.array_equal(s, g["sums"][k])
        if (k + 1) % every == 0:
            np.testing.assert_allclose(net.get(FIELD_V), g["V"][(k + 1) // every - 1], rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(net.get(FIELD_J), g["J_final"], rtol=1e-5, atol=1e-6)


def test_push_and_pull_agree_closed_loop_statistics():
    spec = synthetic.single_block(20000, 100, name="n20k")
    a = Network.from_spec(spec, device=0)
    b = Network.from_spec(spec, device=0)
    sa, _, na = a.run(600, mode="pull")
    sb, _, nb = b.run(600, mode="push")
    # identical for as long as no float-order difference flips a threshold; rates agree overall
    assert abs(sa.sum() - sb.sum()) <= 0.05 * max(sa.sum(), 1) + 5
    assert abs(int(na.sum()) - int(nb.sum())) <= 0.02 * int(na.sum())


# ---------------------------------------------------------------- API behaviour vs oracle

def _oracle_for(spec):
    rowptr, pre, kind, w = O.gen_network(spec.as_dict())
    prop = spec.property()
    return O.OracleBlock(prop, decay_like_reference(prop, spec.dt), rowptr, pre, kind, w, spec.dt, spec.seed)


def test_autotune_and_tuning_knobs():
    from digital_twin_brain_b200._lib import TUNE_CHUNK, TUNE_SCATTER_WORDS
    spec = synthetic.single_block(20000, 100, name="n20k_tune")
    net = Network.from_spec(spec, device=0)
    net.run(60, out=None)
    r = net.autotune(8)
    assert r["scatter_words"] in (1, 2, 4, 8, 16, 32) and r["push_ms"] > 0 and r["pull_ms"] > 0
    assert net.get_tuning(TUNE_SCATTER_WORDS) == r["scatter_words"]
    net.set_tuning(TUNE_CHUNK, 7)
    assert net.get_tuning(TUNE_CHUNK) == 7
    with pytest.raises(Exception):
        net.set_tuning(TUNE_SCATTER_WORDS, 0)


@pytest.mark.parametrize("reverse", [0, 1])
@pytest.mark.parametrize("variant", [0, 1])
@pytest.mark.parametrize("wpw", [1, 4, 32])
def test_scatter_shapes_agree_with_pull_under_forcing(wpw, variant, reverse):
    """One push step from identical state at several launch shapes, register budgets and scatter
    orders vs the exact pull step."""
    from digital_twin_brain_b200._lib import (TUNE_PUSH_METHOD, TUNE_SCATTER_REVERSE, TUNE_SCATTER_VARIANT,
                                              TUNE_SCATTER_WORDS)
    spec = synthetic.single_block(8000, 100, name="n8k")
    a = Network.from_spec(spec, device=0)
    b = Network.from_spec(spec, device=0)
    a.set_tuning(TUNE_PUSH_METHOD, 1)     # the atomic scatter these shapes belong to
    a.set_tuning(TUNE_SCATTER_REVERSE, reverse)
    a.set_tuning(TUNE_SCATTER_WORDS, wpw)
    a.set_tuning(TUNE_SCATTER_VARIANT, variant)
    for _ in range(80):
        a.run(1, mode="push")
        b.run(1, mode="pull")
        # resynchronise b onto a's state so every step starts identical
        b.set(FIELD_V, a.get(FIELD_V)); b.set(FIELD_J, a.get(FIELD_J)); b.set(FIELD_T_LAST, a.get(FIELD_T_LAST))
    np.testing.assert_allclose(a.get(FIELD_J), b.get(FIELD_J), rtol=1e-5, atol=1e-6)


def test_chunked_and_graph_runs_are_identical():
    spec = synthetic.single_block(5000, 50, name="n5k")
    a = Network.from_spec(spec, device=0)
    b = Network.from_spec(spec, device=0)
    sa, ma, na = a.run(100, mode="pull")          # chunks of 32 through CUDA graphs
    rows = [b.run(1, mode="pull") for _ in range(100)]
    assert np.array_equal(sa, np.concatenate([r[0] for r in rows]))
    assert np.array_equal(ma, np.concatenate([r[1] for r in rows]))
    assert np.array_equal(a.get(FIELD_V), b.get(FIELD_V))
    assert np.array_equal(a.get(FIELD_J), b.get(FIELD_J))


def test_per_neuron_noise_isolated_and_oracle():
    spec = synthetic.single_block(3000, 60, noise_rate=0.02, name="n3k")
    net = Network.from_spec(spec, device=0, class_decay=class_decay_like_reference(spec))
    ob = _oracle_for(spec)
    for k in range(120):
        iso = 40 <= k < 60
        rate = None if k % 3 == 0 else 0.015
        s, m, _ = net.run(1, noise_rate=rate, isolated=iso, mode="pull")
        so, mo = ob.run(-1.0 if rate is None else rate, iso)
        assert np.array_equal(s[0], so)
        np.testing.assert_allclose(m[0], mo, rtol=2e-6)
    assert np.array_equal(net.get(FIELD_V), ob.V)
    assert np.array_equal(net.get(FIELD_J), ob.J)


def test_save_load_resume_bit_identical(tmp_path):
    spec = synthetic.single_block(4000, 50, name="n4k")
    net = Network.from_spec(spec, device=0)
    net.run(60, mode="pull")
    ck = str(tmp_path / "ck.bin")
    net.save(ck)
    s1, _, _ = net.run(70, mode="pull")
    v1, j1 = net.get(FIELD_V), net.get(FIELD_J)
    net.load(ck)
    s2, _, _ = net.run(70, mode="pull")
    assert np.array_equal(s1, s2)
    assert np.array_equal(v1, net.get(FIELD_V)) and np.array_equal(j1, net.get(FIELD_J))


def test_scale_property_by_subblock_matches_oracle():
    spec = synthetic.single_block(3000, 60, name="n3k_scale")
    dec = class_decay_like_reference(spec)
    net = Network.from_spec(spec, device=0, class_decay=dec)
    ob = _oracle_for(spec)
    # past the initial refractory period (T_ref = 5 ms = 50 steps), so that the first update
    # after the change shows which I_syn it used
    net.run(120, mode="pull")
    for _ in range(120):
        ob.run(0.01)
    # g_ui of subblock 0 (AMPA) x1.5, GABAa of subblock 1 x0.5 (dist_blockwrapper_pytorch.py:446)
    net.scale_property_by_subblock([0, 1], [10, 12], [1.5, 0.5])
    # the stored I_syn (old parameters) drives the next membrane update, as in models/block.py
    assert np.array_equal(net.get(FIELD_I_SYN), ob.Isyn)
    prop = spec.property()
    base = spec.property()
    prop[prop[:, 3] == 0, 10] = base[prop[:, 3] == 0, 10] * np.float32(1.5)
    prop[prop[:, 3] == 1, 12] = base[prop[:, 3] == 1, 12] * np.float32(0.5)
    ob.P = O.Params.from_property(prop, decay_like_reference(prop, spec.dt))
    for k in range(40):
        s, _, _ = net.run(1, mode="pull")
        so, _ = ob.run(0.01)
        assert np.array_equal(s[0], so)
    assert np.array_equal(net.get(FIELD_V), ob.V)


def test_update_property_across_tile_classes_matches_oracle():
    """Property updates that change which 128-neuron tiles share one parameter class (two
    classes -> per-neuron g_ui, every tile mixed -> two classes again): the update follows
    the new classes, spikes and V bit-identical to the oracle."""
    spec = synthetic.single_block(3000, 60, name="n3k_tiles")
    net = Network.from_spec(spec, device=0, class_decay=class_decay_like_reference(spec))
    ob = _oracle_for(spec)
    base = spec.property()
    mixed = base.copy()
    mixed[:, 10:14] *= np.random.default_rng(5).uniform(0.8, 1.25, (spec.N, 4)).astype(np.float32)
    for prop in (None, mixed, base):
        if prop is not None:
            dec = decay_like_reference(prop, spec.dt)
            net.update_property(prop, np.ascontiguousarray(dec.T))
            ob.update_property(prop, dec)
        for _ in range(80):
            s, _, _ = net.run(1, mode="pull")
            so, _ = ob.run(0.01)
            assert np.array_equal(s[0], so)
        assert np.array_equal(net.get(FIELD_V), ob.V)


def test_update_conn_weight_matches_oracle():
    spec = synthetic.single_block(2000, 40, name="n2k_w")
    net = Network.from_spec(spec, device=0, class_decay=class_decay_like_reference(spec))
    ob = _oracle_for(spec)
    rng = np.random.default_rng(0)
    rows = rng.choice(spec.N, 50, replace=False)
    slot = rng.integers(0, spec.K, 50)
    e = rows * spec.K + slot
    ch = ob.kind[e] + rng.integers(0, 2, 50)
    val = rng.uniform(0.0, 3.0, 50).astype(np.float32)
    net.update_conn_weight(ch, rows, ob.pre[e], val)
    w = ob.w.reshape(-1, 2)
    w[e, ch & 1] = val
    for _ in range(80):
        s, _, _ = net.run(1, mode="pull")
        so, _ = ob.run(0.01)
        assert np.array_equal(s[0], so)
    assert np.array_equal(net.get(FIELD_J), ob.J)
    with pytest.raises(Exception):
        net.update_conn_weight([0], [0], [0], [1.0])  # no self synapse exists


def test_attached_bold_matches_oracle():
    spec = synthetic.single_block(3000, 60, name="n3k_bold")
    net = Network.from_spec(spec, device=0)
    net.attach_bold(np.array([0, 0], np.int32), 1)
    s, _, _ = net.run(300, mode="pull")
    R = 1
    st = [np.zeros(R), np.zeros(R), np.ones(R), np.ones(R)]
    params = dict(epsilon=200, tao_s=0.8, tao_f=0.4, tao_0=1, alpha=0.2, E_0=0.8, V_0=0.02)
    for k in range(300):
        act = np.array([s[k].sum() / spec.N], np.float64)
        out = O.bold_step(np.maximum(act, 1e-5), *st, params, spec.dt / 1000.0)
    # float64 on both sides; device pow and host pow may differ in the last bits
    np.testing.assert_allclose(net.get_bold("bold"), out, rtol=1e-11)
    np.testing.assert_allclose(net.get_bold("q"), st[1], rtol=1e-11)


# ---------------------------------------------------------------- BOLD drop-in

@pytest.mark.parametrize("name,dtype,rtol", [("f32", torch.float32, 2e-5), ("f64", torch.float64, 1e-12)])
def test_bold_drop_in_vs_reference(name, dtype, rtol):
    from digital_twin_brain_b200.models.bold_model_pytorch import BOLD
    g = np.load(os.path.join(GOLDEN, "bold_ref.npz"))
    m = BOLD(epsilon=200, tao_s=0.8, tao_f=0.4, tao_0=1, alpha=0.2, E_0=0.8, V_0=0.02, delta_t=float(g["delta_t"]))
    us = g[f"u_{name}"]
    outs = np.stack([m.run(torch.from_numpy(us[k]).to(dtype)).cpu().numpy() for k in range(len(us))])
    np.testing.assert_allclose(outs, g[f"bold_{name}"], rtol=rtol)
    for f in ("s", "q", "v", "f_in"):
        np.testing.assert_allclose(getattr(m, f).cpu().numpy(), g[f"{f}_{name}"], rtol=rtol, atol=1e-30)


def test_bold_state_update_vs_reference():
    from digital_twin_brain_b200.models.bold_model_pytorch import BOLD
    g = np.load(os.path.join(GOLDEN, "bold_ref.npz"))
    m = BOLD(epsilon=200, tao_s=0.8, tao_f=0.4, tao_0=1, alpha=0.2, E_0=0.8, V_0=0.02, delta_t=float(g["delta_t"]))
    m.state_update(torch.from_numpy(g["su_w"]))
    outs = np.stack([m.run(torch.from_numpy(u)).cpu().numpy() for u in g["su_u"]])
    np.testing.assert_allclose(outs, g["su_bold"], rtol=2e-5)
