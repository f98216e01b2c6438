"""Batched ensembles: members concatenated in one network and stepped by one
kernel per stage equal the same members simulated alone (member-local
generator counters and noise streams), bit for bit in pull mode."""
import numpy as np
import pytest

from oracle import oracle as O
from digital_twin_brain_b200 import Network, synthetic
from digital_twin_brain_b200._lib import FIELD_J, FIELD_T_LAST, FIELD_V

pytestmark = pytest.mark.gpu


def _templates():
    return [synthetic.single_block(5000, 50, gen_seed=21, name="m0"),
            synthetic.whole_brain(R=4, mean_size=1500, sigma=0.4, K=50, gen_seed=22, name="m1"),
            synthetic.single_block(3100, 50, gen_seed=23, name="m2")]


def _scaled(t, f):
    out = synthetic.NetworkSpec(**{k: getattr(t, k) for k in ("name", "region_start", "region_n_exc", "cum", "K",
                                                               "class_property", "gen_seed", "w_scale", "dt", "seed")})
    out.class_property = t.class_property.copy()
    out.class_property[:, 10:14] *= f
    return out


@pytest.mark.parametrize("mode", ["pull", "push"])
def test_batched_members_equal_standalone(mode):
    t = _templates()
    g = np.array([[1, 1, 1, 1], [1.3, 0.7, 1.0, 1.1], [0.6, 1.0, 1.4, 1.0]], np.float32)
    e = synthetic.ensemble(t, g_scale=g)
    ens = Network.from_spec(e, device=0)
    s_e, _, _ = ens.run(150, mode=mode)
    Ve, Je, Te = ens.get(FIELD_V), ens.get(FIELD_J), ens.get(FIELD_T_LAST)
    for m, tm in enumerate(t):
        alone = _scaled(tm, g[m])
        alone.stream_id = m                     # member m's noise stream
        net = Network.from_spec(alone, device=0)
        s_a, _, _ = net.run(150, mode=mode)
        ms = int(e.members["member_start"][m])
        sl = slice(ms, ms + tm.N)
        r0 = synthetic.member_region_index(e, m, 0)
        if mode == "pull":
            assert np.array_equal(Ve[sl], net.get(FIELD_V)), f"member {m}: V differs"
            assert np.array_equal(Je[:, sl], net.get(FIELD_J)), f"member {m}: J differs"
            assert np.array_equal(Te[sl], net.get(FIELD_T_LAST))
            assert np.array_equal(s_e[:, 2 * r0:2 * (r0 + tm.R)], s_a), f"member {m}: spike counts differ"
        else:   # float atomics: rates agree
            assert abs(s_e[:, 2 * r0:2 * (r0 + tm.R)].sum() - s_a.sum()) <= 0.05 * max(s_a.sum(), 1) + 5


def test_ensemble_generator_matches_oracle():
    t = _templates()
    e = synthetic.ensemble(t)
    net = Network.from_spec(e, device=0, build_push=False)
    rp, ix, w = net.get_csr("pull")
    orp, opre, okind, ow = O.gen_network(e.as_dict())
    assert np.array_equal(rp, orp)
    assert np.array_equal(ix, opre | np.where(okind == 2, np.uint32(0x80000000), np.uint32(0)))
    assert np.array_equal(w, ow)


def test_pad_neurons_stay_silent():
    e = synthetic.ensemble(_templates())
    net = Network.from_spec(e, device=0)
    net.run(200, noise_rate=None, mode="push")      # per-neuron noise rates: the pad class has none
    from digital_twin_brain_b200._lib import FIELD_NEW_ACTIVE
    na = net.get(FIELD_NEW_ACTIVE)
    cls = e.neuron_class()
    pad = e.class_property[cls, 3] < 0
    assert pad.any() and not na[pad].any()


def test_many_subblocks_stats_and_bold_match_standalone():
    """300 members: statistics and per-region BOLD run in the multi-CTA k_stats kernel;
    each member still equals the same network simulated alone (in-kernel epilogue)."""
    M = 300
    t = [synthetic.single_block(300, 10, gen_seed=100 + m, name=f"s{m}") for m in range(M)]
    e = synthetic.ensemble(t)
    ens = Network.from_spec(e, device=0, build_push=False)
    ens.attach_bold(e.sub_to_region(), e.R)
    ens.clear_window_spikes()
    s_e, m_e, na_e = ens.run(120, mode="pull")
    win = ens.window_spikes()
    assert np.array_equal(win.astype(np.float64), s_e.sum(0).astype(np.float64))
    bold_e = ens.get_bold("bold")
    for m in (0, 137, M - 1):
        alone = synthetic.single_block(300, 10, gen_seed=100 + m, name="alone")
        alone.stream_id = m
        net = Network.from_spec(alone, device=0, build_push=False)
        net.attach_bold(alone.sub_to_region(), alone.R)
        s_a, m_a, _ = net.run(120, mode="pull")
        r = synthetic.member_region_index(e, m, 0)
        assert np.array_equal(s_e[:, 2 * r:2 * r + 2], s_a)
        assert np.array_equal(m_e[:, 2 * r:2 * r + 2], m_a)
        assert np.array_equal(bold_e[r:r + 1], net.get_bold("bold"))


def test_set_bold_state_roundtrip():
    e = synthetic.ensemble([synthetic.single_block(400, 10, gen_seed=5 + m) for m in range(3)])
    net = Network.from_spec(e, device=0, build_push=False)
    net.attach_bold(e.sub_to_region(), e.R)
    net.run(10, mode="pull")
    for f in ("s", "q", "v", "f_in"):
        v = np.linspace(0.5, 1.5, e.R)
        net.set_bold(f, v)
        assert np.array_equal(net.get_bold(f), v)


def test_ensemble_workload_members_equal_standalone():
    """The batched-ensemble workload (64 members of N~U[5e4,4e5] at 2 % size, per-member g_ui
    factors U[0.5,1.5]): members picked across the ensemble equal themselves simulated alone,
    bit for bit in pull mode."""
    e = synthetic.config_ensemble(scale=0.02)
    members, g = synthetic.ensemble_members(scale=0.02)
    ens = Network.from_spec(e, device=0)
    s_e, m_e, _ = ens.run(120, mode="pull")
    Ve = ens.get(FIELD_V)
    for m in (0, 31, 63):
        alone = _scaled(members[m], g[m])
        alone.stream_id = m
        net = Network.from_spec(alone, device=0)
        s_a, m_a, _ = net.run(120, mode="pull")
        ms = int(e.members["member_start"][m])
        r0 = synthetic.member_region_index(e, m, 0)
        assert np.array_equal(s_e[:, 2 * r0:2 * r0 + 2], s_a), f"member {m}: spike counts differ"
        assert np.array_equal(m_e[:, 2 * r0:2 * r0 + 2], m_a)
        assert np.array_equal(Ve[ms:ms + members[m].N], net.get(FIELD_V)), f"member {m}: V differs"
