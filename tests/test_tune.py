"""Coherent tune analysis on the host side: the peak search
(mbt_tune_peaks) against the reference's identify_tunepeaks and the LON
branch of get_tunepeaks_coherent (tune.c), from the fixture
tests/golden/tune_peaks.npz that tests/golden/make_tune_golden.py made by
running the reference's own functions."""
import os

import numpy as np
import pytest

from mbtrack_b200 import api
from tests.util import GOLDEN


@pytest.fixture(scope="module")
def golden():
    return np.load(os.path.join(GOLDEN, "tune_peaks.npz"))


def test_peak_search_is_the_reference(golden, libmbt):
    nrev = int(golden["nrev"])
    for s, n, v, a in zip(golden["spec"], golden["spec_n"], golden["spec_value"], golden["spec_ampli"]):
        ov, oa, oc = api.tune_peaks(s, nrev)
        assert len(ov) == n
        # a plateau of equal bins gives 0/0 in the parabola: NaN in both
        assert np.array_equal(ov, v[:n], equal_nan=True) and np.array_equal(oa, a[:n])
        assert set(oc.tolist()) <= {1, 2}
    cases = np.concatenate([api.tune_peaks(s, nrev)[2] for s in golden["spec"]])
    assert (cases == 1).any() and (cases == 2).any()      # single-bin peaks and plateaus both seen


def lon_spectrum(x):
    """tune.c:177-197: |DFT| / N of the history, bin 0 halved, normalised by
    the maximum over bins 1 .. N/2 (bin 0 left 0)."""
    n = len(x)
    c = np.abs(np.fft.fft(x))[: n // 2 + 1] / n
    c[0] /= 2
    out = c / c[1:].max()
    out[0] = 0.0
    return out


def test_lon_tunes_match_the_reference(golden, libmbt):
    nt = int(golden["nt"])
    for h, n, v, a in zip(golden["hist"], golden["hist_n"], golden["hist_value"], golden["hist_ampli"]):
        ov, oa, _ = api.tune_peaks(lon_spectrum(h), 1 << nt)
        assert len(ov) == n
        assert np.allclose(ov, v[:n], rtol=1e-12, atol=0) and np.allclose(oa, a[:n], rtol=1e-12, atol=0)


def test_peak_search_arguments(libmbt):
    assert api.lib().mbt_tune_peaks(None, 256, None, None, None, 10) < 0
    v, a, c = api.tune_peaks(np.zeros(129), 256)
    assert len(v) == 0
