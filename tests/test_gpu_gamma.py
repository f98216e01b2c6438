"""Gamma-distributed g_ui (cuda/src/stage/property.cpp:313-471,
dist_blockwrapper_pytorch.py:460 gamma_property_by_subblk) on the device
against the oracle's sampler and the oracle's time step."""
import numpy as np
import pytest

from oracle import oracle as O
from digital_twin_brain_b200 import Network, synthetic
from digital_twin_brain_b200._lib import FIELD_I_SYN, FIELD_V, DtbError
from tests._helpers import decay_like_reference

pytestmark = pytest.mark.gpu


def _spec():
    return synthetic.single_block(3000, 60, name="n3k_gamma")


def test_gamma_draws_match_oracle():
    spec = _spec()
    net = Network.from_spec(spec, device=0)
    sub = spec.property()[:, 3].astype(int)
    net.gamma_property_by_subblock([0, 1, 0], [10, 12, 11], [5.0, 0.5, 50.0], [5.0, 2.0, 10.0])
    g = net.g_factors()
    e, i = np.nonzero(sub == 0)[0], np.nonzero(sub == 1)[0]
    want = np.ones((spec.N, 4), np.float32)
    want[e, 0] = O.gamma(e, 5.0, 5.0, 0, 0, spec.seed)
    want[e, 1] = O.gamma(e, 50.0, 10.0, 1, 0, spec.seed)
    want[i, 2] = O.gamma(i, 0.5, 2.0, 2, 0, spec.seed)
    # device and host log/cos/pow may differ in the last bit of a double: equal after rounding to float
    # except, at most, a rare draw whose accept/reject decision sits on that bit
    same = (g == want) | (np.abs(g - want) <= 1e-6 * np.abs(want))
    assert same.mean() > 0.999
    assert (g[i, 0] == 1).all() and (g[e, 2] == 1).all() and (g[:, 3] == 1).all()
    # a second call draws new values (call counter)
    net.gamma_property_by_subblock([0], [10], [5.0], [5.0])
    g2 = net.g_factors()
    assert not np.array_equal(g2[e, 0], g[e, 0])
    assert np.mean(g2[e, 0] == O.gamma(e, 5.0, 5.0, 0, 1, spec.seed)) > 0.999


def test_gamma_dynamics_and_scaling_match_oracle():
    """The step with per-neuron g_ui is bit-identical to the oracle given the same g values;
    a later subblock scaling multiplies the drawn values (the draws are the new base)."""
    spec = _spec()
    prop = spec.property()
    net = Network.from_spec(spec, device=0)
    net.gamma_property_by_subblock([0, 1], [10, 13], [5.0, 4.0], [5.0, 4.0])
    g = net.g_factors()
    p2 = prop.copy()
    sub = prop[:, 3].astype(int)
    p2[sub == 0, 10] = np.float32(1.0) * g[sub == 0, 0]
    p2[sub == 1, 13] = np.float32(1.0) * g[sub == 1, 3]
    for u in range(4):
        keep = ~(((sub == 0) & (u == 0)) | ((sub == 1) & (u == 3)))
        p2[keep, 10 + u] = prop[keep, 10 + u] * g[keep, u]
    rowptr, pre, kind, w = O.gen_network(spec.as_dict())
    ob = O.OracleBlock(p2, decay_like_reference(p2, spec.dt), rowptr, pre, kind, w, spec.dt, spec.seed)
    for _ in range(150):
        s, _, _ = net.run(1, mode="pull")
        so, _ = ob.run(0.01)
        assert np.array_equal(s[0], so)
    assert np.array_equal(net.get(FIELD_V), ob.V)
    assert np.array_equal(net.get(FIELD_I_SYN), ob.Isyn)
    # x2 on subblock 0 AMPA: column becomes 2 * draw
    net.scale_property_by_subblock([0], [10], [2.0])
    p3 = p2.copy()
    p3[sub == 0, 10] = np.float32(2.0) * g[sub == 0, 0]
    ob.P = O.Params.from_property(p3, decay_like_reference(p3, spec.dt))
    for _ in range(100):
        s, _, _ = net.run(1, mode="pull")
        so, _ = ob.run(0.01)
        assert np.array_equal(s[0], so)
    assert np.array_equal(net.get(FIELD_V), ob.V)


def test_gamma_delta_limit_and_errors():
    spec = _spec()
    net = Network.from_spec(spec, device=0)
    # non-g column: only the near-delta use of simulation/simulation.py:120-144
    with pytest.raises(DtbError):
        net.gamma_property_by_subblock([0], [8], [5.0], [5.0])
    with pytest.raises(DtbError):
        net.gamma_property_by_subblock([0], [3], [1e8], [1e8])
    net.gamma_property_by_subblock([0], [8], [-48.0 * 1e8 * -1], [1e8])   # V_th <- 48 (delta)
    # update_property drops the per-neuron factors
    net.gamma_property_by_subblock([0], [10], [5.0], [5.0])
    net.update_property(spec.property())
    with pytest.raises(DtbError):
        net.g_factors()


def test_graphs_follow_the_update_form():
    """The step's plain form (no gamma g_ui, no I_syn override) and its general form: chunks
    captured in CUDA graphs before gamma factors are drawn, after they are drawn, and after a
    property change (whose next step takes the saved I_syn) give the results of the same run
    without graphs, bit for bit (pull mode)."""
    from digital_twin_brain_b200._lib import FIELD_J, FIELD_T_LAST, TUNE_USE_GRAPHS
    spec = _spec()
    nets = [Network.from_spec(spec, device=0) for _ in range(2)]
    nets[1].set_tuning(TUNE_USE_GRAPHS, 0)
    prop = spec.property().copy()
    prop[:, 10] *= np.float32(1.3)
    for net in nets:
        net.run(64, noise_rate=0.02, mode="pull")                   # plain form, graphs captured
        net.gamma_property_by_subblock([0, 1], [10, 12], [5.0, 0.5], [5.0, 2.0])
        net.run(64, noise_rate=0.02, mode="pull")                   # general form (gamma g_ui)
        net.update_property(prop)                                   # drops the gamma factors
        net.run(64, noise_rate=0.02, mode="pull")                   # override step, then plain
        net.synchronize()
    for f in (FIELD_V, FIELD_J, FIELD_T_LAST, FIELD_I_SYN):
        assert np.array_equal(nets[0].get(f), nets[1].get(f))
