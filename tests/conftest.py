import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")
    config.addinivalue_line("markers", "reference: needs the reference sources (build container only)")


@pytest.fixture(scope="session")
def libmbt():
    from mbtrack_b200 import build as mbuild
    mbuild.build()
    from mbtrack_b200 import api
    return api.lib()


@pytest.fixture(scope="session")
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test selected but no CUDA device is visible")
    return torch.device("cuda:0")


@pytest.fixture(scope="session")
def trained_mlp(cuda_device):
    """The learned field trained once per session with the library's
    standard settings (api.MLP_TRAIN: 1e7 samples of the Faddeeva field),
    as bench.py trains it; returns (network, loss history)."""
    from mbtrack_b200 import api
    m = api.Mlp(seed=31)
    hist = m.train(seed=32, **api.MLP_TRAIN)
    yield m, hist
    m.close()
