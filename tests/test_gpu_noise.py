"""The counter-based noise of the device path (Philox4x32-7 + Box-Muller)
against the reference's generator, statistically: the equilibrium beam
sizes it produces, and reproducibility for a fixed seed."""
import numpy as np
import pytest

from mbtrack_b200 import api
from oracle.binding import Oracle
from tests.util import small_conf

pytestmark = pytest.mark.gpu


def test_equilibrium_sizes_match_reference_generator(tmp_path, cuda_device, libmbt):
    cfg = api.Config(small_conf(tmp_path, "single_bunch.conf", Np=20000, EnableQuantum=1))
    o = Oracle(cfg.params, cfg.bucket, [cfg.params.np_model], cfg.bunch_currents(), cfg.Gl, cfg.Gv, cfg.Gh)
    o.generate_beam()
    t = api.Tracker.from_config(cfg, seed=1234)
    t.load_particles(0, o.get_particles(0))
    o.prepare()
    t.prepare()
    turns = 1500
    so = o.run(turns)
    st = t.run(turns)
    # rms energy spread, bunch length, horizontal and vertical sizes over the
    # last 500 turns: same equilibrium within the statistical error
    for col in (3, 4, 5, 9, 10, 11):
        a = st[-500:, 0, col].mean()
        b = so[-500:, 0, col].mean()
        assert abs(a - b) / b < 0.02, (col, a, b)


def _two_runs(cfg, turns=20):
    runs = []
    for _ in range(2):
        t = api.Tracker.from_config(cfg, seed=99)
        t.generate_beam(7)
        t.prepare()
        runs.append(t.run(turns))
        t.close()
    return runs


def test_philox_is_reproducible(tmp_path, cuda_device, libmbt):
    """Same seed, same beam, same result bit for bit (longitudinal wake
    only: every device reduction has a fixed order)."""
    path = small_conf(tmp_path, "single_bunch.conf", Np=5000, EnableQuantum=1)
    text = open(path).read().replace("plane = HOR", "plane = LON").replace("plane = VER", "plane = LON")
    open(path, "w").write(text)
    cfg = api.Config(path)
    assert cfg.params.planeL == 3 and cfg.params.planeH == 0 and cfg.params.planeV == 0
    a, b = _two_runs(cfg)
    assert np.array_equal(a, b)


def test_transverse_dipole_histograms_reproducible(tmp_path, cuda_device, libmbt):
    """The dipole histograms of the transverse short-range wakes are summed
    as fixed-point integers (order-independent): two runs agree bit for
    bit."""
    cfg = api.Config(small_conf(tmp_path, "single_bunch.conf", Np=5000, EnableQuantum=1))
    assert cfg.params.planeH > 0 or cfg.params.planeV > 0
    a, b = _two_runs(cfg)
    assert np.array_equal(a, b)
