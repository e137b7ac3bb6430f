"""The allocation-free bunch-moments entry point against the regular one.

mbt_bunch_moments_dev_noalloc serves callers that must not allocate device
memory during the call (memory owned by their own pool or framework
allocator, or loops that cannot afford a possibly synchronising cudaMalloc
per call); it keeps its partial sums in a fixed device array inside
libmbt.  This file is collected last so that a failure here stops a `-x`
run only after every other test has run; it also passes on its own in a
fresh process.
"""
import numpy as np
import pytest

from mbtrack_b200 import api
from oracle.binding import Oracle
from tests.golden_cases import Case
from tests.util import stats_err

pytestmark = pytest.mark.gpu


def test_noalloc_matches_regular_on_two_calls(cuda_device, libmbt):
    import torch
    c = Case("feedback_hc")
    o = Oracle(c.params, c.bucket, c.np, c.ib, c.Gl, c.Gv, c.Gh)
    o.generate_beam()
    o.prepare()
    o.run(3)
    p = c.params
    nc = p.ncell
    for ib in (0, c.nb - 1):                      # two calls in a row, different bunches
        X = o.get_particles(ib)
        d = torch.as_tensor(np.ascontiguousarray(X.ravel()), device=cuda_device)
        h_ref = torch.zeros(3 * nc, dtype=torch.float64, device=cuda_device)
        h_new = torch.full((3 * nc,), -1.0, dtype=torch.float64, device=cuda_device)
        ref = api.bunch_moments_dev(int(c.np[ib]), d.data_ptr(), p.sigma_tau, p.nsigma, p.dT, nc,
                                    list(p.track_plane), h_ref.data_ptr())
        new = api.bunch_moments_dev_noalloc(int(c.np[ib]), d.data_ptr(), p.sigma_tau, p.nsigma, p.dT, nc,
                                            list(p.track_plane), h_new.data_ptr())
        assert np.max(stats_err(new, ref)) < 1e-10
        a, b = h_new.cpu().numpy().reshape(3, nc), h_ref.cpu().numpy().reshape(3, nc)
        assert np.array_equal(a[0], b[0])                       # counts, bit for bit
        scale = max(np.max(np.abs(X[1])), np.max(np.abs(X[2]))) * c.np[ib]
        assert np.max(np.abs(a[1:] - b[1:])) <= 1e-13 * scale


def test_noalloc_rejects_oversized_histograms(cuda_device, libmbt):
    import torch
    d = torch.zeros(6 * 64, dtype=torch.float64, device=cuda_device)
    h = torch.zeros(3 * 2048, dtype=torch.float64, device=cuda_device)
    with pytest.raises(api.MbtError) as e:
        api.bunch_moments_dev_noalloc(64, d.data_ptr(), 1e-11, 5.0, 0.04, 2048, [1, 1, 1], h.data_ptr())
    assert e.value.code == -1


def test_noalloc_largest_histogram_caps_the_blocks(cuda_device, libmbt):
    """The largest histogram (ncell = 1024, the accepted limit) over 1e6
    macroparticles: the fixed array holds 83 block records where the regular
    path uses 489, so the partial sums are grouped differently.  Two calls
    in a row; counts identical, sums and statistics equal to rounding."""
    import torch
    rng = np.random.default_rng(5)
    n, nc, sgm, nsig = 1_000_000, 1024, 1e-11, 5.0
    dT = 2.0 * nsig / nc
    X = rng.normal(size=(6, n)) * np.array([sgm, 1e-4, 1e-5, 1e-3, 1e-5, 1e-6])[:, None]
    X[1] += 3e-6
    X[2] -= 2e-7
    d = torch.as_tensor(np.ascontiguousarray(X.ravel()), device=cuda_device)
    for _ in range(2):
        h_ref = torch.zeros(3 * nc, dtype=torch.float64, device=cuda_device)
        h_new = torch.full((3 * nc,), -1.0, dtype=torch.float64, device=cuda_device)
        ref = api.bunch_moments_dev(n, d.data_ptr(), sgm, nsig, dT, nc, [1, 1, 1], h_ref.data_ptr())
        new = api.bunch_moments_dev_noalloc(n, d.data_ptr(), sgm, nsig, dT, nc, [1, 1, 1], h_new.data_ptr())
        assert np.max(stats_err(new, ref)) < 1e-10
        a, b = h_new.cpu().numpy().reshape(3, nc), h_ref.cpu().numpy().reshape(3, nc)
        assert a[0].sum() > 0.99 * n
        assert np.array_equal(a[0], b[0])
        scale = np.max(np.abs(X[1:3])) * n
        assert np.max(np.abs(a[1:] - b[1:])) <= 1e-13 * scale
