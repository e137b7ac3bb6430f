"""The CPU oracle (oracle/mbt_oracle.c) against fixtures produced by the
reference's own sources: every case must agree bit for bit."""
import numpy as np
import pytest

from oracle.binding import Oracle
from tests.golden_cases import CASES, Case


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_fixture(name):
    c = Case(name)
    o = Oracle(c.params, c.bucket, c.np, c.ib, c.Gl, c.Gv, c.Gh)
    o.generate_beam()
    init = c.bunch_slices(c.init)
    for i in range(c.nb):
        assert np.array_equal(o.get_particles(i), init[i]), "initial distribution, bunch %d" % i
    assert np.array_equal(o.prepare(), c.init_stats)
    if c.deviates.size:
        st, dev = o.run(c.turns, record=True)
        assert np.array_equal(dev[:c.deviates.size], c.deviates)
    else:
        st = o.run(c.turns)
    assert np.array_equal(st, c.stats)
    final = c.bunch_slices(c.final)
    for i in range(c.nb):
        assert np.array_equal(o.get_particles(i), final[i]), "final coordinates, bunch %d" % i
    v, ph = o.state(0)
    assert np.array_equal(v, c.vrf_phi)
    assert np.array_equal(ph, c.phasor)


def test_oracle_injected_deviates_reproduce_generator():
    """Feeding the oracle's own deviates back gives the same run."""
    c = Case("single_noise")
    a = Oracle(c.params, c.bucket, c.np, c.ib, c.Gl, c.Gv, c.Gh)
    b = Oracle(c.params, c.bucket, c.np, c.ib, c.Gl, c.Gv, c.Gh)
    for o in (a, b):
        o.generate_beam()
        o.prepare()
    sa, dev = a.run(c.turns, record=True)
    sb = b.run(c.turns, dev_in=dev)
    assert np.array_equal(sa, sb)
    assert np.array_equal(a.get_particles(0), b.get_particles(0))
