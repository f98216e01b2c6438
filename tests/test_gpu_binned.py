"""Binned push (DTB_TUNE_PUSH_METHOD = 2): firing rows append their synaptic events to
per-destination bins that the next update adds in shared memory.  It must give the
sums of the reference's push (cuda/src/stage/presynaptic_voltage.cpp:152-266) and of
models/block.py's sparse product, to float32 rounding: checked against the exact pull
step from identical state, against the reference's golden run under teacher forcing,
with bins that overflow into the atomic fallback, at every bin size, across method
switches, checkpoints and state reads while events wait in the bins."""
import os

import numpy as np
import pytest

from digital_twin_brain_b200 import Network, synthetic
from digital_twin_brain_b200._lib import (FIELD_I_SYN, FIELD_J, FIELD_STEP, FIELD_T, FIELD_T_LAST, FIELD_V, TUNE_BIN_CAPACITY,
                                          TUNE_BIN_SHIFT, TUNE_BIN_WORDS, TUNE_PUSH_METHOD, TUNE_STAGE_WAIT_LIMIT,
                                          TUNE_STEP_VARIANT, DtbError)
from tests._helpers import GOLDEN, unpack
from tests.test_gpu_parity import class_decay_like_reference

pytestmark = pytest.mark.gpu

ATOMIC, BINNED = 1, 2


def _resync(dst, src):
    dst.set(FIELD_V, src.get(FIELD_V))
    dst.set(FIELD_J, src.get(FIELD_J))
    dst.set(FIELD_T_LAST, src.get(FIELD_T_LAST))


def _binned(spec, tune=None):
    net = Network.from_spec(spec, device=0)
    net.set_tuning(TUNE_PUSH_METHOD, BINNED)
    for k, v in (tune or {}).items():
        net.set_tuning(k, v)
    return net


@pytest.mark.parametrize("variant", [0, 3])
@pytest.mark.parametrize("words", [1, 64, 256])
@pytest.mark.parametrize("shift", [10, 11, 13])
def test_binned_step_equals_pull_step_from_same_state(shift, words, variant):
    """One binned push step from identical state vs the exact pull step, 60 times (past the
    50-step refractory window, so spikes, thresholds and t_last are exercised).  Step
    variant 3 with 1024-neuron bins is the staged update that adds the bins into the staged
    J planes (a partial last tile, and a last chunk with a warp that has no tile: N = 9000);
    with larger bins it runs the unstaged fold."""
    spec = synthetic.single_block(9000, 100, noise_rate=0.02, name="n9k")
    a = _binned(spec, {TUNE_BIN_SHIFT: shift, TUNE_BIN_WORDS: words, TUNE_STEP_VARIANT: variant})
    b = Network.from_spec(spec, device=0)
    for _ in range(60):
        a.run(1, mode="push")
        b.run(1, mode="pull")
        np.testing.assert_allclose(a.get(FIELD_J), b.get(FIELD_J), rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(a.get(FIELD_V), b.get(FIELD_V), rtol=1e-5, atol=1e-5)
        assert np.array_equal(a.get(FIELD_T_LAST), b.get(FIELD_T_LAST))
        _resync(b, a)


@pytest.mark.parametrize("variant", [0, 2, 3])
@pytest.mark.parametrize("cap", [1, 2])
def test_bins_overflowing_into_atomics(cap, variant):
    """Capacities far below the events per bin: most events take the atomic fallback; dense
    activity (p = 0.3) keeps every bin full (unstaged and staged update)."""
    spec = synthetic.whole_brain(R=5, mean_size=900, sigma=0.5, K=80, gen_seed=4, name="wb5_k80")
    a = _binned(spec, {TUNE_BIN_CAPACITY: cap, TUNE_STEP_VARIANT: variant})
    b = Network.from_spec(spec, device=0)
    for k in range(40):
        rate = 0.3 if k % 2 else 0.05
        a.run(1, noise_rate=rate, mode="push")
        b.run(1, noise_rate=rate, mode="pull")
        np.testing.assert_allclose(a.get(FIELD_J), b.get(FIELD_J), rtol=1e-5, atol=1e-5)
        _resync(b, a)


@pytest.mark.parametrize("variant", [0, 3])
def test_binned_teacher_forced_vs_reference_golden(variant):
    """The reference's own block.py run (golden fixture), its spikes fed to the binned push."""
    g = np.load(os.path.join(GOLDEN, "single_block_2k.npz"))
    spec = synthetic.config_single_block()
    net = Network.from_spec(spec, device=0, build_push=True, class_decay=class_decay_like_reference(spec))
    net.set_tuning(TUNE_PUSH_METHOD, BINNED)
    net.set_tuning(TUNE_STEP_VARIANT, variant)
    act_ref = unpack(g["active"], spec.N)
    nact_ref = unpack(g["new_active"], spec.N)
    every = int(g["v_every"])
    for k in range(int(g["steps"])):
        s, _ = net.step_forced(act_ref[k], nact_ref[k], noise_rate=0.01, mode="push")
        assert np.array_equal(s, g["sums"][k])
        if (k + 1) % every == 0:
            np.testing.assert_allclose(net.get(FIELD_V), g["V"][(k + 1) // every - 1], rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(net.get(FIELD_J), g["J_final"], rtol=1e-5, atol=1e-6)


def test_pending_bins_across_switches_reads_and_checkpoints(tmp_path):
    """Events waiting in the bins reach J before anything else reads it: a state read, a pull
    run, the atomic push, a checkpoint, a property change; identical runs stay identical."""
    spec = synthetic.whole_brain(R=4, mean_size=3000, sigma=0.4, K=60, gen_seed=8, name="wb4")
    a = _binned(spec)
    b = _binned(spec)
    sa, _, _ = a.run(70, mode="push")      # graph chunks of 32 + a tail
    sb = np.concatenate([b.run(1, mode="push")[0] for _ in range(70)])
    # the order of the float additions varies from run to run: rates agree
    assert abs(float(sa.sum()) - float(sb.sum())) <= 0.05 * max(float(sa.sum()), 1.0) + 3
    assert np.array_equal(sa[:50], sb[:50])    # nobody leaves the initial refractory window before step 50
    # switch: pull, atomic push, binned again
    ref = Network.from_spec(spec, device=0)
    _resync(ref, a)
    ref.set(FIELD_T, a.get(FIELD_T))
    ref.set(FIELD_STEP, a.get(FIELD_STEP))
    a.run(5, mode="pull")
    ref.run(5, mode="pull")
    assert np.array_equal(a.get(FIELD_V), ref.get(FIELD_V)) and np.array_equal(a.get(FIELD_J), ref.get(FIELD_J))
    a.run(3, mode="push")
    a.set_tuning(TUNE_PUSH_METHOD, ATOMIC)
    a.run(3, mode="push")
    a.set_tuning(TUNE_PUSH_METHOD, BINNED)
    a.run(4, mode="push")
    # checkpoint with events pending, then the same steps twice
    ck = str(tmp_path / "ck.bin")
    a.save(ck)
    s1, _, _ = a.run(20, mode="push")
    a.load(ck)
    s2, _, _ = a.run(20, mode="push")
    assert abs(float(s1.sum()) - float(s2.sum())) <= 0.05 * max(float(s1.sum()), 1.0) + 3
    # a parameter change keeps the current I_syn, computed from the folded J
    a.run(2, mode="push")
    isyn = a.get(FIELD_I_SYN)
    a.scale_property_by_subblock([0], [10], [1.3])
    np.testing.assert_array_equal(a.get(FIELD_I_SYN), isyn)


def test_autotune_chooses_a_push_method():
    spec = synthetic.single_block(30000, 100, name="n30k_tune")
    net = Network.from_spec(spec, device=0)
    net.run(60, out=None)
    r = net.autotune(6)
    pm = net.get_tuning(TUNE_PUSH_METHOD)
    assert pm in (ATOMIC, BINNED) and r["push_ms"] > 0
    net.run(10, mode="push")


@pytest.mark.parametrize("how", ["atomic", "binned", "rows", "slots", "masks", "stream"])
def test_synaptic_event_count_every_method(how):
    """FIELD_EVENTS advances by the out-degree sum of every neuron that propagated (spike | noise),
    whichever kernel propagates (the scatters count the rows they push, the gathers the entries
    they add)."""
    from digital_twin_brain_b200._lib import FIELD_EVENTS, FIELD_NEW_ACTIVE, TUNE_PULL_METHOD
    spec = synthetic.whole_brain(R=3, mean_size=2000, sigma=0.3, K=40, gen_seed=6, name="wb3_ev")
    net = Network.from_spec(spec, device=0)
    mode = "push" if how in ("atomic", "binned") else "pull"
    if how == "binned":
        net.set_tuning(TUNE_PUSH_METHOD, BINNED)
    elif mode == "pull":
        net.set_tuning(TUNE_PULL_METHOD, {"rows": 1, "slots": 2, "masks": 3, "stream": 4}[how])
    qrp = net.get_csr_rowptr("push")
    outdeg = np.diff(qrp)
    for n in (1, 3, 40):
        for _ in range(n):
            e0 = net.get(FIELD_EVENTS)
            net.run(1, noise_rate=0.03, mode=mode)
            na = net.get(FIELD_NEW_ACTIVE).astype(bool)
            assert net.get(FIELD_EVENTS) - e0 == int(outdeg[na].sum())


def test_binned_staged_copy_given_up():
    """The staged binned update with the completion-wait limit at 0: every warp gives up on
    its first copy, loads its tiles from global memory into the other buffer, the fold adds
    the bins there, the run reports DTB_ERR_CUDA each step, and the results match the exact
    pull step from the same state."""
    spec = synthetic.single_block(9000, 100, noise_rate=0.02, name="n9k")
    a = _binned(spec, {TUNE_STEP_VARIANT: 3, TUNE_STAGE_WAIT_LIMIT: 0})
    b = Network.from_spec(spec, device=0)
    for _ in range(60):
        with pytest.raises(DtbError) as e:
            a.run(1, mode="push")
        assert e.value.code == 2 and "staged state copy did not complete" in str(e.value)
        b.run(1, mode="pull")
        np.testing.assert_allclose(a.get(FIELD_J), b.get(FIELD_J), rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(a.get(FIELD_V), b.get(FIELD_V), rtol=1e-5, atol=1e-5)
        assert np.array_equal(a.get(FIELD_T_LAST), b.get(FIELD_T_LAST))
        _resync(b, a)
    a.set_tuning(TUNE_STAGE_WAIT_LIMIT, 1 << 20)
    a.run(5, mode="push")
    a.synchronize()
