"""Checkpoint and resume on the GPU: a run saved after some turns and
resumed in a fresh context continues as the uninterrupted run (coordinates,
statistics, RF state; the Philox noise is keyed by the turn), and a damaged
or foreign checkpoint is refused with the context untouched.

Bit for bit in every case: the device reductions have a fixed order, and
the dipole histograms of the transverse short-range wakes are fixed-point
integer sums, which do not depend on the order of the atomics."""
import numpy as np
import pytest

from mbtrack_b200 import api
from tests.golden_cases import Case

pytestmark = pytest.mark.gpu


def _tracker(c, seed=5):
    t = api.Tracker(c.params, c.bucket, c.np, c.ib, c.Gl, c.Gv, c.Gh, seed=seed)
    t.generate_beam(11)
    t.prepare()
    return t


@pytest.mark.parametrize("name", ["train_rw_hom", "feedback_hc", "single_noise"])
def test_resume_continues_bit_for_bit(tmp_path, cuda_device, name):
    c = Case(name)
    ck = str(tmp_path / "run.ckpt")
    a = _tracker(c)
    a.run(7)
    a.checkpoint_save(ck)
    assert api.checkpoint_check(ck) == (7, c.nb)
    sa = a.run(9)
    ca = a.get_all()
    a.close()
    b = _tracker(c)
    b.run(3)                       # a different state, overwritten by the load
    b.checkpoint_load(ck)
    sb = b.run(9)
    cb = b.get_all()
    b.close()
    assert np.array_equal(sa, sb)
    assert np.array_equal(ca, cb)


def test_bad_checkpoints_leave_the_context_untouched(tmp_path, cuda_device):
    c = Case("train_rw_hom")
    ck = tmp_path / "run.ckpt"
    a = _tracker(c)
    a.run(4)
    a.checkpoint_save(str(ck))
    data = ck.read_bytes()
    bad = tmp_path / "bad.ckpt"
    bad.write_bytes(data[:len(data) // 2])
    ref = _tracker(c)
    ref.run(6)
    want = ref.run(5)
    ref.close()
    b = _tracker(c)
    b.run(6)
    with pytest.raises(api.MbtError) as e:
        b.checkpoint_load(str(bad))
    assert e.value.code == -8
    # another seed: a foreign configuration
    other = _tracker(c, seed=6)
    with pytest.raises(api.MbtError) as e:
        other.checkpoint_load(str(ck))
    assert e.value.code == -5
    other.close()
    got = b.run(5)
    b.close()
    a.close()
    assert np.array_equal(got, want)
