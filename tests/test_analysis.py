"""Growth-rate analysis of the per-turn statistics (mbtrack_b200.analysis)."""
import numpy as np

from mbtrack_b200 import analysis


def test_growth_rate_of_a_synthetic_instability():
    turns = np.arange(800)
    rng = np.random.default_rng(3)
    k = 0.021
    # noise floor and an exponentially growing mode, added in quadrature,
    # saturating
    amp = np.sqrt(1e-14 + (1e-7 * np.exp(k * (turns - 300))) ** 2)
    amp = np.minimum(amp, 5e-5) * (1.0 + 1e-3 * rng.normal(size=len(turns)))
    stats = np.zeros((len(turns), 4, 12))
    for b in range(4):
        stats[:, b, 2] = amp * (1 if b % 2 else -1)
    a = analysis.centroid_amplitude(stats, "VER")
    assert np.allclose(a, amp)
    w = analysis.exponential_window(a)
    assert w is not None and 300 < w[0] < 360 and w[1] < 580
    assert abs(analysis.growth_rate(a, w) - k) < 0.02 * k


def test_no_window_without_growth():
    a = 1e-7 * (1.0 + 1e-2 * np.random.default_rng(1).normal(size=500))
    assert analysis.exponential_window(a) is None
