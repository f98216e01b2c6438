"""Spike statistics restated from analysis/spike_statistics.py and getpsd.py, against the reference outputs."""
import os

import numpy as np

from digital_twin_brain_b200 import analysis as A
from tests._helpers import GOLDEN


def test_statistics_match_reference():
    g = np.load(os.path.join(GOLDEN, "statistics_ref.npz"))
    r = g["raster"]
    assert A.mean_firing_rate(r) == float(g["rate"])
    np.testing.assert_array_equal(A.instantaneous_rate(r), g["inst"])
    np.testing.assert_allclose(A.coefficient_of_variation(r), float(g["cv"]), rtol=1e-12)
    f, p = A.spike_psd(r)
    np.testing.assert_array_equal(f, g["psd_f"])
    np.testing.assert_allclose(p, g["psd"], rtol=1e-6)
    wf, wp = A.get_psd(g["sig"], fs=1000, resolution=0.5)
    np.testing.assert_array_equal(wf, g["welch_f"])
    np.testing.assert_allclose(wp, g["welch"], rtol=1e-12)
