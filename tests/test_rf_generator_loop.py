"""The generator loop of the RF feedback (an extension: [rf_feedback]
generator_gain, loop_delay) in the oracle.  With gain 0 it is the
reference's full correction (the golden fixture, bit for bit, in
test_oracle_golden.py); with a gain so large that G / (1 + G) rounds to
one and no delay it gives the reference's run again; with gain 10 and a
one-turn delay the RF phasor lags the full correction, so the run differs
but stays close to it."""
import numpy as np

from oracle.binding import Oracle
from tests.golden_cases import Case
from tests.util import stats_err


def _run(c, gain, delay):
    p = c.params.copy() if hasattr(c.params, "copy") else c.params
    p.rffb_gain, p.rffb_delay = gain, delay
    o = Oracle(p, c.bucket, c.np, c.ib, c.Gl, c.Gv, c.Gh)
    o.generate_beam()
    o.prepare()
    if c.deviates.size:
        st = o.run(c.turns, dev_in=c.deviates)
    else:
        st = o.run(c.turns)
    return st, o.state(0)[0]


def test_infinite_gain_without_delay_is_the_reference_feedback():
    c = Case("feedback_hc")
    assert c.params.rffb == 1
    st, v = _run(c, 1e300, 0)
    assert np.max(stats_err(st, c.stats)) < 1e-12
    assert np.max(np.abs(v - c.vrf_phi) / np.abs(c.vrf_phi)) < 1e-12


def test_gain_ten_one_turn_delay_lags_the_full_correction():
    c = Case("feedback_hc")
    st, v = _run(c, 10.0, 1)
    assert np.all(np.isfinite(st))
    d = np.max(stats_err(st, c.stats))
    assert 1e-12 < d < 1e-2, d                       # a different, nearby run
    assert np.max(np.abs(v - c.vrf_phi) / np.abs(c.vrf_phi)) < 1e-2
