"""Gamma-distributed property draws (cuda/src/stage/property.cpp:313-471): the
oracle's Marsaglia-Tsang sampler against the Gamma distribution itself."""
import numpy as np
import pytest
from scipy import stats

from oracle import oracle as O


@pytest.mark.parametrize("alpha,beta", [(0.5, 2.0), (1.0, 1.0), (5.0, 5.0), (50.0, 10.0)])
def test_gamma_distribution(alpha, beta):
    x = O.gamma(np.arange(40_000), alpha, beta, receptor=1, call=3, seed=11).astype(np.float64)
    assert (x >= 0).all()
    # Kolmogorov-Smirnov against Gamma(alpha, rate=beta)
    ks = stats.kstest(x, stats.gamma(a=alpha, scale=1.0 / beta).cdf)
    assert ks.pvalue > 1e-3, ks
    assert abs(x.mean() / (alpha / beta) - 1) < 0.02
    assert abs(x.var() / (alpha / beta ** 2) - 1) < 0.05


def test_gamma_streams():
    n = np.arange(1000)
    a = O.gamma(n, 5.0, 5.0, 0, 0, 1)
    assert np.array_equal(a, O.gamma(n, 5.0, 5.0, 0, 0, 1))           # deterministic
    assert not np.array_equal(a, O.gamma(n, 5.0, 5.0, 1, 0, 1))       # receptor changes the stream
    assert not np.array_equal(a, O.gamma(n, 5.0, 5.0, 0, 1, 1))       # so does the call number
    assert np.array_equal(O.gamma(n, 0.0, 2.0, 0, 0, 1), np.zeros(1000, np.float32))
    # the reference's near-delta use (alpha = value * 1e8, beta = 1e8) gives the value
    d = O.gamma(n, 0.7 * 1e8, 1e8, 2, 0, 1)
    assert np.abs(d / 0.7 - 1).max() < 1e-3
