"""The update kernel with staged state loads (bulk copies one tile ahead into
shared memory, DTB_TUNE_STEP_VARIANT = 2) computes exactly what the plain
update computes, including a partial last tile and an odd neuron count."""
import numpy as np
import pytest

from digital_twin_brain_b200 import Network, synthetic
from digital_twin_brain_b200._lib import (FIELD_ACTIVE, FIELD_I_SYN, FIELD_J, FIELD_T_LAST, FIELD_V, TUNE_CHUNK,
                                          TUNE_PULL_METHOD, TUNE_STEP_VARIANT)

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("variant", [2, 3, 4])
@pytest.mark.parametrize("N", [3002, 3001, 128 * 40], ids=["partial_tile", "odd_n", "whole_tiles"])
def test_staged_update_equals_plain(N, variant):
    spec = synthetic.single_block(N, 60, name=f"staged_{N}")
    nets = []
    for variant in (0, variant):
        net = Network.from_spec(spec, device=0)
        net.set_tuning(TUNE_STEP_VARIANT, variant)
        net.set_tuning(TUNE_CHUNK, 1)            # every step starts with the plain (gather-free) update
        net.set_tuning(TUNE_PULL_METHOD, 1)
        nets.append(net)
    for n in (1, 60, 90):
        outs = [net.run(n, noise_rate=0.05, mode="pull") for net in nets]
        for x, y in zip(outs[0], outs[1]):
            assert np.array_equal(x, y)
        for f in (FIELD_V, FIELD_J, FIELD_T_LAST, FIELD_I_SYN, FIELD_ACTIVE):
            assert np.array_equal(nets[0].get(f), nets[1].get(f))
    for net in nets:
        net.synchronize()                      # raises if a staged copy timed out
    assert outs[0][2].sum() > 0


@pytest.mark.parametrize("variant", [2, 3])
def test_staged_copy_wait_given_up_falls_back_exactly(variant):
    """With the completion-wait limit at 0 the update gives up on every staged copy at once (a
    bounded device-side wait that runs out; nothing faults or hangs): it loads that state from
    global memory, stops staging, drains the copy before exiting, and the run reports
    DTB_ERR_CUDA once while its results stay bit-identical to the plain update's."""
    from digital_twin_brain_b200._lib import TUNE_STAGE_WAIT_LIMIT, DtbError
    spec = synthetic.single_block(128 * 300 + 17, 60, name="staged_giveup")
    ref = Network.from_spec(spec, device=0)
    net = Network.from_spec(spec, device=0)
    for n in (ref, net):
        n.set_tuning(TUNE_CHUNK, 1)
        n.set_tuning(TUNE_PULL_METHOD, 1)
    ref.set_tuning(TUNE_STEP_VARIANT, 0)
    net.set_tuning(TUNE_STEP_VARIANT, variant)
    net.set_tuning(TUNE_STAGE_WAIT_LIMIT, 0)
    errors = 0
    for _ in range(80):
        ref.run(1, noise_rate=0.05, mode="pull")
        try:
            net.run(1, noise_rate=0.05, mode="pull")
        except DtbError as e:
            assert e.code == 2 and "staged state copy did not complete" in str(e)
            errors += 1
    assert errors == 80                        # every step gave up, and reported it once
    for f in (FIELD_V, FIELD_J, FIELD_T_LAST, FIELD_I_SYN, FIELD_ACTIVE):
        assert np.array_equal(ref.get(f), net.get(f))
    net.set_tuning(TUNE_STAGE_WAIT_LIMIT, 1 << 20)
    net.run(5, noise_rate=0.05, mode="pull")    # staging again, no error left behind
    net.synchronize()
