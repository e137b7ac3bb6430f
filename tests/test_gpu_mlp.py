"""The learned field network on a B200: tensor-core forward pass and
gradient against the CPU restatement (oracle/mlp_oracle.c, same operand
roundings), and the trained network against the Faddeeva field with the
north star's tolerance (1e-4 relative field error)."""
import numpy as np
import pytest
import torch

from mbtrack_b200 import api
from oracle import binding

pytestmark = pytest.mark.gpu

BLOCKS = {"W1": (0, 384), "b1": (384, 512), "W2": (512, 16896), "b2": (16896, 17024), "W3": (17024, 33408),
          "b3": (33408, 33536), "W4": (33536, 33792), "b4": (33792, 33794)}


def inputs(n, seed):
    rng = np.random.default_rng(seed)
    return np.stack([rng.uniform(0, 8, n), rng.uniform(0, 8, n), rng.uniform(0.05, 1, n)], 1).astype(np.float32)


def perturbed(m, seed):
    """Weights with non-zero biases, so every parameter block is exercised."""
    p = m.params()
    rng = np.random.default_rng(seed)
    for name in ("b1", "b2", "b3", "b4"):
        lo, hi = BLOCKS[name]
        p[lo:hi] = rng.normal(0, 0.2, hi - lo)
    m.set_params(p)
    return p


def test_forward_matches_oracle(cuda_device):
    m = api.Mlp(seed=3)
    p = perturbed(m, 4)
    x = inputs(1000, 5)     # 8 tiles, the last one partial
    xd = torch.as_tensor(x, device="cuda")
    out = torch.zeros((len(x), 2), dtype=torch.float32, device="cuda")
    m.forward_dev(len(x), xd.data_ptr(), out.data_ptr())
    ref = binding.mlp_forward(p, x)
    got = out.cpu().numpy()
    # BF16 activations keep 8 significant bits; the GPU's hardware tanh and
    # the oracle's libm tanh can round to neighbouring BF16 values, and such
    # a difference of 2^-8 in one activation propagates: a few 1e-3 of the
    # output scale at most
    scale = np.abs(ref).max()
    assert np.max(np.abs(got - ref)) <= 1e-2 * scale, np.max(np.abs(got - ref)) / scale
    assert np.median(np.abs(got - ref)) <= 2e-3 * scale


def test_gradient_matches_oracle(cuda_device):
    m = api.Mlp(seed=6)
    p = perturbed(m, 7)
    x = inputs(300, 8)      # 3 tiles, the last one partial
    t = np.random.default_rng(9).normal(0.8, 0.2, (300, 2)).astype(np.float32)
    xd, td = torch.as_tensor(x, device="cuda"), torch.as_tensor(t, device="cuda")
    g, loss = m.gradient_dev(len(x), xd.data_ptr(), td.data_ptr())
    gr, lr = binding.mlp_gradient(p, x, t)
    assert loss == pytest.approx(lr, rel=1e-2)
    for name, (lo, hi) in BLOCKS.items():
        norm = np.linalg.norm(gr[lo:hi])
        assert norm > 0, name
        assert np.linalg.norm(g[lo:hi] - gr[lo:hi]) <= 2e-2 * norm, (name, np.linalg.norm(g[lo:hi] - gr[lo:hi]) / norm)


def field_points(n, seed, kind):
    """Offsets and rms sizes of elliptic Gaussians [m]: offsets uniform in
    the network's box (|a|, |b| < 8) or Gaussian with twice the rms size,
    aspect ratios uniform or log-uniform (flat beams), a third of them with
    sy > sx."""
    rng = np.random.default_rng(seed)
    sx = rng.uniform(2e-5, 3e-4, n)
    r = 0.05 * 20 ** rng.random(n) if kind == "flat" else rng.uniform(0.05, 1.0, n)
    sy = sx * r
    if kind == "box":
        dx, dy = rng.uniform(-7.99, 7.99, n) * sx, rng.uniform(-7.99, 7.99, n) * sy
    else:
        dx, dy = rng.normal(0, 2, n) * sx, rng.normal(0, 2, n) * sy
    sw = rng.random(n) < 0.3
    return (np.where(sw, dy, dx), np.where(sw, dx, dy), np.where(sw, sy, sx), np.where(sw, sx, sy))


@pytest.mark.parametrize("kind", ["box", "core", "flat"])
def test_trained_field_within_the_tolerance(cuda_device, trained_mlp, kind):
    """The network trained with the standard settings against the Faddeeva
    field (mbt_gauss_field_dev, FP64) on 2e6 held-out points: relative error
    of the field vector |F_net - F| / |F| at most 1e-4 (the north star's
    bar) everywhere.  What the network gains over the method without it:
    the quadrature envelope alone (network output 0) is within 2e-4 of the
    field, the trained network at least 10 times closer at its worst point."""
    m, hist = trained_mlp
    assert np.all(np.isfinite(hist)) and hist[-100:].mean() < 0.01 * hist[:5].mean()
    n = 2_000_000
    arrs = [torch.as_tensor(a, device="cuda") for a in field_points(n, 17, kind)]
    ptr = [a.data_ptr() for a in arrs]
    f, g, e = [[torch.empty(n, dtype=torch.float64, device="cuda") for _ in range(2)] for _ in range(3)]
    assert api.lib().mbt_gauss_field_dev(n, *ptr, f[0].data_ptr(), f[1].data_ptr(), None) == 0
    torch.cuda.synchronize()
    fallbacks = m.field_dev(n, *ptr, g[0].data_ptr(), g[1].data_ptr())
    zero = api.Mlp(seed=1)
    zero.set_params(np.zeros(api.MLP_NPARAM, dtype=np.float32))
    zero.field_dev(n, *ptr, e[0].data_ptr(), e[1].data_ptr())
    zero.close()
    F = torch.hypot(f[0], f[1])
    err = (torch.hypot(g[0] - f[0], g[1] - f[1]) / F).cpu().numpy()
    err0 = (torch.hypot(e[0] - f[0], e[1] - f[1]) / F).cpu().numpy()
    print("%s: learned field max %.2e p99.9 %.2e median %.2e; envelope alone max %.2e; %d outside the domain"
          % (kind, err.max(), np.percentile(err, 99.9), np.median(err), err0.max(), fallbacks))
    assert np.all(np.isfinite(err))
    assert err.max() <= 1e-4
    assert err.max() <= 0.1 * err0.max()
