"""Device w(z) and Bassetti-Erskine field (mbt_wofz_dev, mbt_be_field_dev)
against the oracle, plus the reference's known answers."""
import numpy as np
import pytest

from mbtrack_b200 import api
from oracle import binding
from tests.test_wofz import KNOWN

pytestmark = pytest.mark.gpu


def _dev(a, dev):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a), device=dev)


def test_wofz_known_answers_and_grid(cuda_device, libmbt):
    import torch
    rng = np.random.default_rng(2)
    x = np.concatenate([[k[0] for k in KNOWN], rng.uniform(-8, 8, 20000), rng.uniform(-0.5, 0.5, 2000),
                        rng.uniform(-40, 40, 2000)])
    y = np.concatenate([[k[1] for k in KNOWN], rng.uniform(-8, 8, 20000), rng.uniform(-0.5, 0.5, 2000),
                        rng.uniform(-40, 40, 2000)])
    dx, dy = _dev(x, cuda_device), _dev(y, cuda_device)
    re = torch.empty_like(dx)
    im = torch.empty_like(dx)
    fl = torch.empty(x.size, dtype=torch.int32, device=cuda_device)
    api.wofz_dev(dx.data_ptr(), dy.data_ptr(), re.data_ptr(), im.data_ptr(), x.size, fl.data_ptr())
    torch.cuda.synchronize()
    r, i, f = re.cpu().numpy(), im.cpu().numpy(), fl.cpu().numpy()
    for k, (_, _, kr, ki, tol) in enumerate(KNOWN):
        assert abs(r[k] - kr) <= tol and abs(i[k] - ki) <= tol
    orr, oi, of = binding.wofz(x, y)
    assert np.array_equal(f, of)
    ok = of == 1
    mag = np.maximum(np.hypot(orr[ok], oi[ok]), 1e-300)
    assert np.max(np.abs(r[ok] - orr[ok]) / mag) < 1e-13
    assert np.max(np.abs(i[ok] - oi[ok]) / mag) < 1e-13


def test_be_field_against_oracle(cuda_device, libmbt):
    import torch
    rng = np.random.default_rng(3)
    sx, sz = 0.2, 0.012      # mm
    dx = rng.normal(0, 3 * sx * 1e-3, 5000)
    dy = rng.normal(0, 3 * sz * 1e-3, 5000)
    factdq = 1.7e3
    ex = torch.empty(dx.size, dtype=torch.float64, device=cuda_device)
    ey = torch.empty_like(ex)
    a, b = _dev(dx, cuda_device), _dev(dy, cuda_device)
    api.be_field_dev(a.data_ptr(), b.data_ptr(), dx.size, sx, sz, factdq, ex.data_ptr(), ey.data_ptr())
    torch.cuda.synchronize()
    rx, ry = binding.be_field(dx, dy, sx, sz, factdq)
    scale = np.max(np.hypot(rx, ry))
    assert np.max(np.abs(ex.cpu().numpy() - rx)) / scale < 1e-12
    assert np.max(np.abs(ey.cpu().numpy() - ry)) / scale < 1e-12
