"""The field every beam-ion kick uses (orc_gauss_field, the oracle of
mbt_gauss_field_dev) and the oracle's beam-ion stage, on the CPU.

The Bassetti-Erskine branch is pinned to the reference's own field
expression (fbi_weakstrong.c:155-191, restated bit for bit by
orc_be_field_n and pinned to the reference through the w(z) golden grid);
the near-round branch to the closed form of the round Gaussian."""
import math
import os

import numpy as np
import pytest

from oracle import binding
from oracle.binding import Oracle
from mbtrack_b200 import api
from tests.util import small_conf

SQRT_PI = math.sqrt(math.pi)


def ref_unit_field(dx, dy, sx, sy):
    """The reference's Ex, Ey for factdQ = 1, scaled to a unit line charge."""
    ex, ey = binding.be_field(dx, dy, sx * 1e3, sy * 1e3, 1.0)
    fbe = math.sqrt(2.0 * (sx * sx - sy * sy))
    return -ex / (SQRT_PI * fbe), -ey / (SQRT_PI * fbe)


def test_flat_beam_matches_reference_expression():
    rng = np.random.default_rng(7)
    for sx, sy in ((1e-4, 1e-5), (2e-4, 1.5e-4), (5e-5, 4.9e-5), (1e-3, 5e-5)):
        dx = rng.uniform(0, 8 * sx, 400)
        dy = rng.uniform(0, 8 * sy, 400)
        gx, gy = binding.gauss_field(dx, dy, sx, sy)
        rx, ry = ref_unit_field(dx, dy, sx, sy)
        scale = np.max(np.hypot(rx, ry))
        assert np.max(np.abs(gx - rx)) <= 1e-13 * scale
        assert np.max(np.abs(gy - ry)) <= 1e-13 * scale


def test_symmetries_and_swap():
    rng = np.random.default_rng(8)
    dx, dy = rng.normal(0, 3e-4, 200), rng.normal(0, 3e-5, 200)
    gx, gy = binding.gauss_field(dx, dy, 1e-4, 1e-5)
    mx, my = binding.gauss_field(-dx, -dy, 1e-4, 1e-5)
    assert np.array_equal(gx, -mx) and np.array_equal(gy, -my)
    # sy > sx: axes swapped
    sx_, sy_ = binding.gauss_field(dy, dx, 1e-5, 1e-4)
    assert np.array_equal(sx_, gy) and np.array_equal(sy_, gx)


def test_round_limit_and_far_field():
    s = 1e-4
    r = np.linspace(0.01, 12, 60) * s
    th = np.linspace(0.1, 1.4, 60)
    dx, dy = r * np.cos(th), r * np.sin(th)
    gx, gy = binding.gauss_field(dx, dy, s, s)
    exact = -np.expm1(-r * r / (2 * s * s)) / (math.pi * r * r)
    assert np.allclose(gx, dx * exact, rtol=1e-13, atol=0)
    assert np.allclose(gy, dy * exact, rtol=1e-13, atol=0)
    # far from the beam: a line charge plus the quadrupole term
    # (sx^2 - sy^2) / x^2 of the elliptic profile (next order (s/x)^4)
    far = 60 * s
    fx, fy = binding.gauss_field(np.array([far]), np.array([0.0]), 2 * s, s)
    assert fx[0] == pytest.approx((1.0 + 3 * s * s / far ** 2) / (math.pi * far), rel=5e-6)
    assert abs(fy[0]) < 1e-200   # the two exponentials cancel to rounding


def test_branch_continuity_at_round_ratio():
    rng = np.random.default_rng(9)
    dx, dy = rng.uniform(0, 4e-4, 100), rng.uniform(0, 4e-4, 100)
    sx = 1e-4
    a = binding.gauss_field(dx, dy, sx, 0.995 * sx)            # Bassetti-Erskine
    b = binding.gauss_field(dx, dy, sx, 0.995 * sx * (1 + 1e-9))  # quadrature
    scale = np.max(np.hypot(*a))
    assert np.max(np.abs(a[0] - b[0])) < 1e-8 * scale
    assert np.max(np.abs(a[1] - b[1])) < 1e-8 * scale


def test_oracle_stage_is_deterministic_and_acts(tmp_path):
    """Two oracle runs agree exactly; the clouds grow along the train; with
    no gas the stage leaves the beam alone."""
    conf = small_conf(tmp_path, "beam_ion.conf", Np=60, filling="SINGLE10", NrevTot=4)
    C = api.Config(conf)
    bi = C.beam_ion()
    bi.n_ip, bi.ions_per_passage, bi.pressure = 3, 40, 1e-6
    out = []
    for pressure in (bi.pressure, bi.pressure, 0.0):
        bi.pressure = pressure
        o = Oracle(C.params, C.bucket, np.full(C.nbunch, 60), C.bunch_currents())
        o.generate_beam()
        o.prepare()
        o.enable_beam_ion(bi)
        st = o.run(3)
        out.append((st, o.beam_ion_clouds(), [o.get_particles(i) for i in range(C.nbunch)]))
    (s1, c1, p1), (s2, c2, p2), (s0, c0, p0) = out
    assert np.array_equal(s1, s2) and np.array_equal(c1, c2)
    assert all(np.array_equal(a, b) for a, b in zip(p1, p2))
    ions = c1[:, :, 0]
    assert np.all(ions[:, 0] == 0) and np.all(np.diff(ions, axis=1) > 0)
    assert np.all(c0[:, :, 0] == 0)
    o = Oracle(C.params, C.bucket, np.full(C.nbunch, 60), C.bunch_currents())
    o.generate_beam()
    o.prepare()
    ref = o.run(3)
    assert np.array_equal(ref, s0)
