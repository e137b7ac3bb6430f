"""Checkpoint and resume on the GPU: a run saved after some turns and
resumed in a fresh context continues as the uninterrupted run (coordinates,
statistics, RF state; the Philox noise is keyed by the turn), and a damaged
or foreign checkpoint is refused with the context untouched.

Bit for bit where the run itself repeats bit for bit.  With transverse
short-range wakes the particle pass sums the dipole histograms with
shared-memory atomics, whose order varies, so two uninterrupted runs already
differ in the last bits; there the resumed run must agree with the
uninterrupted one as closely as two uninterrupted runs agree (statistics
1e-10 of the rms, coordinates 1e-12 of the spread, the smoke test's bounds)."""
import numpy as np
import pytest

from mbtrack_b200 import api
from tests.golden_cases import Case
from tests.util import coord_err, stats_err

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
    if c.params.planeV == 0 and c.params.planeH == 0:
        assert np.array_equal(sa, sb)
        assert np.array_equal(ca, cb)
    else:
        assert float(np.max(stats_err(sb, sa))) < 1e-10
        assert float(np.max(coord_err(cb, ca))) < 1e-12


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
