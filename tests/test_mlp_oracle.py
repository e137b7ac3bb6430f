"""The CPU restatement of the learned field network (oracle/mlp_oracle.c)
against the same network in plain FP64 (numpy): the restatement rounds the
operands and activations to BF16 as the tensor-core kernels do, so the two
agree to BF16 accuracy, and its gradient matches a finite difference of
its own loss direction to first order."""
import numpy as np

from oracle import binding


def _params(seed):
    rng = np.random.default_rng(seed)

    def glorot(fi, fo, n):
        return rng.uniform(-1, 1, n) * np.sqrt(6.0 / (fi + fo))
    p = np.zeros(33794, np.float32)
    p[0:384] = glorot(3, 128, 384)
    p[384:512] = rng.normal(0, 0.2, 128)
    p[512:16896] = glorot(128, 128, 16384)
    p[16896:17024] = rng.normal(0, 0.2, 128)
    p[17024:33408] = glorot(128, 128, 16384)
    p[33408:33536] = rng.normal(0, 0.2, 128)
    p[33536:33792] = glorot(128, 2, 256)
    p[33792:] = rng.normal(0, 0.2, 2)
    return p


def _fp64_network(p, x):
    def gelu(z):     # sigmoid form z sigma(1.702 z)
        return z / (1 + np.exp(-1.702 * z))
    f = np.stack([x[:, 0] / 4 - 1, x[:, 1] / 4 - 1, 1 + 2 * np.log(x[:, 2]) / np.log(20)], 1).astype(float)
    W1, b1 = p[0:384].reshape(128, 3), p[384:512]
    W2, b2 = p[512:16896].reshape(128, 128), p[16896:17024]
    W3, b3 = p[17024:33408].reshape(128, 128), p[33408:33536]
    W4, b4 = p[33536:33792].reshape(2, 128), p[33792:]
    h = gelu(f @ W1.T + b1)
    h = gelu(h @ W2.T + b2)
    h = gelu(h @ W3.T + b3)
    return h @ W4.T + b4


def test_bf16_restatement_follows_the_fp64_network():
    rng = np.random.default_rng(2)
    x = np.stack([rng.uniform(0, 8, 300), rng.uniform(0, 8, 300), rng.uniform(0.05, 1, 300)], 1).astype(np.float32)
    p = _params(1)
    got = binding.mlp_forward(p, x)
    ref = _fp64_network(p.astype(float), x)
    scale = np.abs(ref).max()
    # BF16 keeps 8 significant bits (relative rounding 2^-9 per step)
    assert np.max(np.abs(got - ref)) <= 1e-2 * scale
    assert np.median(np.abs(got - ref)) <= 2e-3 * scale


def test_restated_gradient_is_a_descent_direction():
    rng = np.random.default_rng(3)
    x = np.stack([rng.uniform(0, 8, 64), rng.uniform(0, 8, 64), rng.uniform(0.05, 1, 64)], 1).astype(np.float32)
    t = rng.normal(0.5, 0.2, (64, 2)).astype(np.float32)
    p = _params(4)
    g, loss = binding.mlp_gradient(p, x, t)
    assert np.isfinite(g).all() and np.linalg.norm(g) > 0
    out = binding.mlp_forward(p, x)
    assert abs(loss - float(np.mean(np.sum((out.astype(float) - t) ** 2, 1)) * 1)) <= 1e-6 * max(loss, 1.0) * 64
    step = 1e-2 / np.linalg.norm(g)
    _, loss2 = binding.mlp_gradient((p - step * g).astype(np.float32), x, t)
    assert loss2 < loss

