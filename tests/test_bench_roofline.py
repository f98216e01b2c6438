"""bench.py's roofline bookkeeping (CPU only): which kernels a method's step has, their
algorithmic bytes per launch, and the step's bytes against the step model
B_step = N*44 + S_touched*13 + N/8."""
import math
import os
import sys

import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


class _Spec:
    N, S, K = 1_000_000, 100_000_000, 100


PEAKS = {"hbm_gbs": 6500.0}


def _kt(evs=1e6, upd=0.05, prop=0.04):
    return {"events_per_step": evs, "update_ms": upd, "propagate_ms": prop, "step_ms": upd + prop}


def test_push_atomic_kernels_and_step_model():
    r, step = bench.roofline_of(_Spec, _kt(), "push", 1, 0, PEAKS)
    assert set(step["kernels"]) == {"update", "scatter"}
    N, evs = _Spec.N, 1e6
    assert math.isclose(step["bytes_per_step_model"], N * 44 + evs * 13 + N / 8)
    assert r["kernel"] == "update" and r["peak"] == 6500.0
    assert math.isclose(r["frac"], r["achieved"] / 6500.0)


def test_push_binned_kernels():
    _, step = bench.roofline_of(_Spec, _kt(), "push", 2, 0, PEAKS)
    assert set(step["kernels"]) == {"update+fold", "binned scatter"}


@pytest.mark.parametrize("method,ordered", [(0, True), (-1, True), (1, False), (2, True), (3, True), (4, False)])
def test_pull_method_labels(method, ordered):
    """Low activity: auto (0) and slots/masks run the ordered push (two kernels); rows and the
    streamed gather are one fused kernel whatever the activity."""
    _, step = bench.roofline_of(_Spec, _kt(evs=1e6), "pull", 1, method, PEAKS)
    if ordered:
        assert set(step["kernels"]) == {"slots+update", "ordered scatter"}
    else:
        assert set(step["kernels"]) == {"gather+update"}


def test_pull_auto_at_high_activity_is_fused():
    # 20 % of the neurons propagating: auto leaves the ordered push for the streamed gather
    _, step = bench.roofline_of(_Spec, _kt(evs=0.2 * _Spec.N * _Spec.K), "pull", 1, 0, PEAKS)
    assert set(step["kernels"]) == {"gather+update"}
