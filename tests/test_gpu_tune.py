"""Coherent tune spectra on the GPU (mbt_tune_spectra_dev) against numpy's
FFT of the same histories, the reference's LON tunes through the GPU
spectra (tests/golden/tune_peaks.npz), and the betatron tunes of a tracked
bunch (mbtrack_b200.analysis.coherent_tunes)."""
import os

import numpy as np
import pytest
import torch

from mbtrack_b200 import analysis, api
from tests.test_tune import lon_spectrum
from tests.util import GOLDEN, small_conf

pytestmark = pytest.mark.gpu


def padded_spectrum(x):
    """tune.c:240-276: |FFT| of the history zero-padded to 2N, bins 0 .. N-1
    normalised by their maximum (bin 0 the real part)."""
    n = len(x)
    f = np.fft.fft(np.concatenate([x, np.zeros(n)]))[:n]
    m = np.abs(f)
    m[0] = abs(f[0].real)
    return m / m.max()


def gpu_spectra(h, plane):
    x = torch.as_tensor(np.ascontiguousarray(h), dtype=torch.float64, device="cuda")
    n = h.shape[1]
    out = torch.zeros((h.shape[0], n // 2 + 1 if plane == 0 else n), dtype=torch.float64, device="cuda")
    api.tune_spectra_dev(x.data_ptr(), n, h.shape[0], n, plane, out.data_ptr(), None)
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("nturn", [4, 64, 512, 2048])
def test_spectra_match_numpy(nturn, cuda_device):
    rng = np.random.default_rng(nturn)
    t = np.arange(nturn)
    h = np.stack([np.cos(2 * np.pi * rng.uniform(0, 0.5) * t) * np.exp(-t / 900) + 0.1 * rng.normal(size=nturn)
                  + rng.uniform(-1, 1) for _ in range(7)])
    for plane, ref in ((0, lon_spectrum), (1, padded_spectrum), (2, padded_spectrum)):
        got = gpu_spectra(h, plane)
        want = np.stack([ref(x) for x in h])
        assert np.max(np.abs(got - want)) < 1e-12, (plane, np.max(np.abs(got - want)))


def test_reference_lon_tunes_through_the_gpu(cuda_device):
    g = np.load(os.path.join(GOLDEN, "tune_peaks.npz"))
    spec = gpu_spectra(g["hist"], 0)
    for s, n, v, a in zip(spec, g["hist_n"], g["hist_value"], g["hist_ampli"]):
        ov, oa, _ = api.tune_peaks(s, g["hist"].shape[1])
        assert len(ov) == n
        assert np.allclose(ov, v[:n], rtol=1e-9, atol=0) and np.allclose(oa, a[:n], rtol=1e-9, atol=0)


def test_limits_are_errors(cuda_device):
    x = torch.zeros(8192, dtype=torch.float64, device="cuda")
    with pytest.raises(api.MbtError):
        api.tune_spectra_dev(x.data_ptr(), 4096, 1, 4096, 1, x.data_ptr())      # padded beyond 2048
    with pytest.raises(api.MbtError):
        api.tune_spectra_dev(x.data_ptr(), 100, 1, 100, 0, x.data_ptr())        # not a power of two


def test_betatron_tunes_of_a_tracked_bunch(tmp_path, cuda_device, libmbt):
    """A displaced bunch (noise off) oscillates at its fractional betatron
    tunes, QH0 = 18.17 and QV0 = 10.23, moved by chromaticity and the wakes
    by far less than one bin (1 / 1024)."""
    cfg = api.Config(small_conf(tmp_path, "single_bunch.conf", Np=20000, xxCM_offset=0.3, zzCM_offset=0.3))
    t = api.Tracker.from_config(cfg)
    t.generate_beam(5)
    t.prepare()
    st = t.run(512)
    t.close()
    for plane, q in (("HOR", 0.17), ("VER", 0.23)):
        peaks = analysis.coherent_tunes(st, plane)[0]
        assert peaks, plane
        top = max(peaks, key=lambda p: p[1])
        assert abs(top[0] - q) < 2.0 / 1024, (plane, peaks)
