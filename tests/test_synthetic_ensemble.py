"""The batched-ensemble workload spec (CPU): member sizes, per-member g_ui factors and the
concatenated layout (members on 128-neuron tiles, one BOLD region per member)."""
import numpy as np

from digital_twin_brain_b200 import synthetic


def test_ensemble_workload_spec():
    members, g = synthetic.ensemble_members()
    assert len(members) == 64 and g.shape == (64, 4)
    sizes = np.array([m.N for m in members])
    assert sizes.min() >= 50_000 and sizes.max() <= 400_000
    assert (g >= 0.5).all() and (g <= 1.5).all()
    assert len({m.gen_seed for m in members}) == 64
    e = synthetic.config_ensemble(scale=0.01)
    ms = e.members["member_start"]
    assert (ms % 128 == 0).all() and len(ms) == 64
    small, gs = synthetic.ensemble_members(scale=0.01)
    assert np.array_equal(g, gs)
    # g_ui of member m's classes = template g_ui x its factors
    for m in (0, 17, 63):
        r = synthetic.member_region_index(e, m, 0)
        row = e.class_property[2 * r]
        np.testing.assert_allclose(row[10:14], small[m].class_property[0, 10:14] * gs[m], rtol=1e-6)
        assert row[3] == 2 * r
    assert e.N >= sum(m.N for m in small)
