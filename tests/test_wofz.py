"""w(z) of the oracle: the known answers of the reference's own test
(test_complexerrf.c:33-59), a grid evaluated by the reference's
complex_errorfunc_wofz_algo680 (bit for bit), and identities of w."""
import math
import os

import numpy as np
import pytest

from oracle import binding

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# (x, y, re, im, tolerance): test_complexerrf.c:33-59
KNOWN = [
    (0.0, 0.0, 1.0, 0.0, 1e-8),
    (0.01, 0.01, 0.9887176929549547, 0.01108529605747726, 1e-8),
    (0.5, 0.5, 0.5331567079121750, 0.2304882313844584, 1e-8),
    (0.5, 1.0, 0.391234, 0.127202, 1e-5),
    (1.0, 1.0, 0.3047442052569128, 0.2082189382028316, 1e-8),
    (2.5, 2.5, 0.1167371250446503, 0.1079085859964814, 1e-8),
    (15.0, 15.0, 0.01882714532513676, 0.01878535427799565, 1e-8),
]


@pytest.mark.parametrize("x,y,re,im,tol", KNOWN)
def test_known_answers(x, y, re, im, tol):
    r, i, f = binding.wofz([x], [y])
    assert f[0] == 1
    assert abs(r[0] - re) <= tol and abs(i[0] - im) <= tol


def test_reference_grid_bit_exact():
    z = np.load(os.path.join(GOLDEN, "wofz_grid.npz"))
    r, i, f = binding.wofz(z["x"], z["y"])
    assert np.array_equal(f, z["flag"])
    ok = z["flag"] == 1
    assert np.array_equal(r[ok], z["re"][ok])
    assert np.array_equal(i[ok], z["im"][ok])


def test_imaginary_axis_is_scaled_erfc():
    # w(iy) = exp(y^2) erfc(y) for real y >= 0
    ys = np.linspace(0.0, 5.0, 51)
    r, i, _ = binding.wofz(np.zeros_like(ys), ys)
    ref = np.array([math.exp(y * y) * math.erfc(y) for y in ys])
    assert np.max(np.abs(r - ref) / ref) < 5e-13
    assert np.all(i == 0.0)


def test_reflection_symmetry():
    # w(-conj(z)) = conj(w(z))
    rng = np.random.default_rng(1)
    x, y = rng.uniform(-6, 6, 500), rng.uniform(-6, 6, 500)
    r1, i1, f1 = binding.wofz(x, y)
    r2, i2, f2 = binding.wofz(-x, y)
    ok = (f1 == 1) & (f2 == 1)
    assert np.allclose(r1[ok], r2[ok], rtol=1e-14, atol=1e-300)
    assert np.allclose(i1[ok], -i2[ok], rtol=1e-14, atol=1e-300)


def test_be_field_reference_convention():
    """Round-beam limit and sign: the field points away from the centre."""
    dx = np.array([1e-5, -1e-5, 0.0, 0.0])
    dy = np.array([0.0, 0.0, 1e-5, -1e-5])
    ex, ey = binding.be_field(dx, dy, 0.2, 0.02, 1.0)
    assert ex[0] == -ex[1] and ey[2] == -ey[3]
    assert np.sign(ex[0]) != np.sign(ex[1])
