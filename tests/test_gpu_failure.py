"""Failure reporting on the GPU without a device fault: the sticky device
error word, set from the host, makes the next run fail with the code its
bit stands for (the path a kernel's bounded wait takes when it gives up),
and a wait that nothing ends gives up after its bound and is reported."""
import pytest

from mbtrack_b200 import api
from mbtrack_b200.abi import MBT_ERR_STATE, MBT_ERR_TIMEOUT
from tests.golden_cases import Case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("bits,code,words", [(4, MBT_ERR_TIMEOUT, "tensor cores"), (2, MBT_ERR_TIMEOUT, "pipeline"),
                                             (1, MBT_ERR_STATE, "deviates")])
def test_error_word_fails_the_next_run(cuda_device, bits, code, words):
    c = Case("feedback_hc")
    t = api.Tracker(c.params, c.bucket, c.np, c.ib, c.Gl, c.Gv, c.Gh)
    t.generate_beam(3)
    t.prepare()
    t.run(2)                                  # healthy
    t.inject_device_error(bits)
    with pytest.raises(api.MbtError) as e:
        t.run(1)
    assert e.value.code == code and words in str(e.value), str(e.value)
    t.close()
    # a fresh context on the same device is unaffected
    u = api.Tracker(c.params, c.bucket, c.np, c.ib, c.Gl, c.Gv, c.Gh)
    u.generate_beam(3)
    u.prepare()
    assert u.run(2).shape[0] == 2
    u.close()


def test_bounded_wait_gives_up_and_reports(cuda_device):
    L = api.lib()
    assert L.mbt_selftest_bounded_wait(256, None) == MBT_ERR_TIMEOUT
    # the device is still usable after the wait gave up
    import torch
    x = torch.arange(1000, dtype=torch.float64, device=cuda_device)
    assert float(x.sum()) == 499500.0
