"""Growth of coupled-bunch motion from the per-turn statistics of a run
(the arrays mbt_run_turns returns: turns x bunches x 12, columns as in
mbt.h: centroid LON, HOR, VER, rms ..., slope centroid ..., slope rms ...).

The beam-ion instability shows as an exponential rise of the bunch
centroids along the train out of the sampling noise of the initial beam.
Its growth rate is the slope of the logarithm of the coherent part of the
centroid amplitude (the initial level removed in quadrature, as the noise
and the growing mode are uncorrelated) over the turns where that rise is
exponential: after the start-up and before saturation.
"""
import numpy as np

PLANE_COLUMN = {"LON": 0, "HOR": 1, "VER": 2}


def centroid_amplitude(stats, plane="VER"):
    """rms over bunches of the centroid of `plane`, per turn."""
    s = np.asarray(stats)
    c = s[:, :, PLANE_COLUMN[plane]]
    return np.sqrt((c * c).mean(axis=1))


def exponential_window(amp, start_factor=2.0, stop_fraction=0.3, baseline_turns=50):
    """Turns [first, last] of the exponential rise of `amp`: from where it
    first exceeds start_factor times its initial level (median of the first
    baseline_turns) to where it first reaches stop_fraction of its maximum.
    None when the amplitude never rises that far."""
    a = np.asarray(amp, dtype=float)
    base = np.median(a[:baseline_turns])
    top = stop_fraction * a.max()
    if top <= start_factor * base:
        return None
    above = np.nonzero(a > start_factor * base)[0]
    first = int(above[0])
    reach = np.nonzero(a[first:] >= top)[0]
    if len(reach) == 0:
        return None
    last = first + int(reach[0])
    if last - first < 10:
        return None
    return first, last


def growth_rate(amp, window, baseline_turns=50):
    """Least-squares slope (per turn) of log sqrt(amp^2 - base^2) over the
    turns of `window`, base the initial level (median of the first
    baseline_turns)."""
    a = np.asarray(amp, dtype=float)
    base = np.median(a[:baseline_turns])
    first, last = window
    turns = np.arange(first, last + 1)
    coh = np.sqrt(np.maximum(a[first:last + 1] ** 2 - base * base, 1e-300))
    return float(np.polyfit(turns, np.log(coh), 1)[0])


def coherent_tunes(stats, plane="VER", nturn=None, max_peaks=10):
    """Coherent tunes of every bunch from the centroid history of `plane`
    (get_tunepeaks_coherent and identify_tunepeaks of tune.c, the spectra on
    the GPU): the last nturn turns (a power of two; the largest one that
    fits by default).  Returns per bunch a list of (tune, amplitude) with the
    tune as a fraction of the revolution frequency; for HOR and VER the
    reference's value (bin / nturn of the spectrum zero-padded to 2 nturn)
    is halved to give that fraction."""
    import torch
    from . import api
    s = np.asarray(stats)
    n = nturn or 1 << int(np.floor(np.log2(s.shape[0])))
    hist = np.ascontiguousarray(s[-n:, :, PLANE_COLUMN[plane]].T)
    pl = PLANE_COLUMN[plane]
    nout = n // 2 + 1 if pl == 0 else n
    x = torch.as_tensor(hist, dtype=torch.float64, device="cuda")
    spec = torch.zeros((hist.shape[0], nout), dtype=torch.float64, device="cuda")
    api.tune_spectra_dev(x.data_ptr(), n, hist.shape[0], n, pl, spec.data_ptr(), None)
    torch.cuda.synchronize()
    out = []
    for row in spec.cpu().numpy():
        v, a, _ = api.tune_peaks(row, n, max_peaks)
        out.append([(float(t) / (1.0 if pl == 0 else 2.0), float(m)) for t, m in zip(v, a)])
    return out
