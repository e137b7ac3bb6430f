"""Per-step entry point mbt_bunch_moments_dev (weak_bunch_mean_rms +
fnp_ring_update binning on caller-owned device data) against the oracle."""
import numpy as np
import pytest

from mbtrack_b200 import api
from oracle.binding import Oracle
from tests.golden_cases import Case
from tests.util import stats_err

pytestmark = pytest.mark.gpu


def test_bunch_moments_match_oracle(cuda_device, libmbt):
    import torch
    c = Case("feedback_hc")
    o = Oracle(c.params, c.bucket, c.np, c.ib, c.Gl, c.Gv, c.Gh)
    o.generate_beam()
    o.run(0)
    init_stats = o.prepare()
    p = c.params
    nc = p.ncell
    for ib in range(c.nb):
        X = o.get_particles(ib)
        d = torch.as_tensor(np.ascontiguousarray(X.ravel()), device=cuda_device)
        h = torch.zeros(3 * nc, dtype=torch.float64, device=cuda_device)
        st = api.bunch_moments_dev(int(c.np[ib]), d.data_ptr(), p.sigma_tau, p.nsigma, p.dT, nc,
                                   list(p.track_plane), h.data_ptr())
        assert np.max(stats_err(st, init_stats[ib])) < 1e-10
        hist = h.cpu().numpy().reshape(3, nc)
        ring = o.histograms(ib)
        assert np.array_equal(hist[0], ring[3])          # counts, bit for bit
        scale = np.max(np.abs(X[1])) * c.np[ib]
        assert np.max(np.abs(hist[1] - ring[4])) <= 1e-13 * scale
