"""Live pin of the oracle against the reference's own sources (compiled
unmodified into oracle/_ref/libmbtref.so).  Needs the reference tree, so it
runs in the build container; the committed fixtures carry the same pin to
machines without it (tests/test_oracle_golden.py)."""
import os

import numpy as np
import pytest

from oracle import binding
from oracle.binding import Oracle, Reference
from tests.util import small_conf

pytestmark = pytest.mark.skipif(not (binding.reference_available() or os.path.exists(binding.REF_SO)),
                                reason="reference sources not present")


def _pair(path):
    R = Reference(path)
    p = R.params()
    st0 = R.prepare()
    p = R.params()
    Gl, Gv, Gh, _ = R.greens()
    O = Oracle(p, R.bucket, R.np, R.ib, Gl, Gv, Gh)
    O.generate_beam()
    assert np.array_equal(O.prepare(), st0)
    return R, O


@pytest.mark.parametrize("conf,over,turns", [
    ("single_bunch.conf", {"Np": 600, "xxCM_offset": 0.05, "EnableQuantum": 1}, 15),
    ("uniform_fill.conf", {"Np": 40, "Nmlt": 2, "xxCM_offset": 0.05}, 3),
    ("feedback_hc.conf", {}, 12),
])
def test_oracle_is_the_reference(tmp_path, conf, over, turns):
    R, O = _pair(small_conf(tmp_path, conf, **over))
    sr = R.run(turns)
    so = O.run(turns)
    assert np.array_equal(sr, so)
    for i in range(R.nb):
        assert np.array_equal(R.get_particles(i), O.get_particles(i))
        assert np.array_equal(R.ampinv(i), O.ampinv(i))
    assert np.array_equal(R.state(0)[0], O.state(0)[0])


@pytest.mark.parametrize("scan", [
    {"scan_type": 1, "Nscan": 3, "NrevScan": 4, "scan_start": 120.0, "scan_step": 40.0},
    {"scan_type": 3, "Nscan": 2, "NrevScan": 30},
])
def test_oracle_is_the_reference_through_scan_steps(tmp_path, scan):
    """Current and Q-factor scans (tracking_scan_step_worker tracking.c:43-57,
    worker_weakweak.c:388-393) with long-range resistive wall, its 50-kick
    trigger (restarted at every boundary) and a longitudinal resonator:
    bit-identical across the scan boundaries."""
    from tests.util import add_section, add_tracking_keys
    path = small_conf(tmp_path, "uniform_fill.conf", Np=40, Nmlt=2, filling="SINGLE10", xxCM_offset=0.05,
                      NrevTot=1)
    add_tracking_keys(path, triggerRW=1)
    R, O = _pair(add_section(path, "scan", **scan))
    turns = scan["Nscan"] * scan["NrevScan"]
    assert np.array_equal(R.run(turns), O.run(turns))
    for i in range(R.nb):
        assert np.array_equal(R.get_particles(i), O.get_particles(i))
    assert np.array_equal(R.state(0)[0], O.state(0)[0])


def test_oracle_is_the_reference_with_short_range_rw(tmp_path):
    """Short-range resistive wall in three planes on top of the broadband
    resonators (the reference's Green's functions given to the oracle)."""
    from tests.util import rw_short_conf
    R, O = _pair(rw_short_conf(tmp_path, Np=500, xxCM_offset=0.05, zzCM_offset=0.02))
    assert np.array_equal(R.run(20), O.run(20))
    assert np.array_equal(R.get_particles(0), O.get_particles(0))
