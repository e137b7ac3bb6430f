"""The beam-ion stage on a B200 against the oracle's restatement of the same
model (oracle/mbt_oracle.c, beam_ion): the field function, and whole turns
of a bunch train with ion clouds at several interaction points."""
import numpy as np
import pytest
import torch

from mbtrack_b200 import api
from oracle import binding
from oracle.binding import Oracle
from tests.util import coord_err, small_conf, stats_err

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")


def test_gauss_field_matches_oracle(cuda_device):
    rng = np.random.default_rng(11)
    n = 4000
    sx = rng.uniform(2e-5, 3e-4, n)
    ratio = np.concatenate([rng.uniform(0.02, 1.0, n - 800), rng.uniform(0.99, 1.0, 400),
                            rng.uniform(1.0, 20.0, 400)])
    sy = sx * ratio
    dx = rng.normal(0, 4, n) * sx
    dy = rng.normal(0, 4, n) * sy
    dx[:50] = 0.0
    dy[50:100] = 0.0
    gx, gy = torch.empty(n, dtype=torch.float64, device="cuda"), torch.empty(n, dtype=torch.float64, device="cuda")
    inputs = [dev(a) for a in (dx, dy, sx, sy)]      # kept alive until the kernel has run
    L = api.lib()
    rc = L.mbt_gauss_field_dev(n, *[a.data_ptr() for a in inputs], gx.data_ptr(), gy.data_ptr(), None)
    assert rc == 0
    torch.cuda.synchronize()
    ox, oy = binding.gauss_field(dx, dy, sx, sy)
    scale = np.hypot(ox, oy).max()
    assert np.max(np.abs(gx.cpu().numpy() - ox)) <= 1e-12 * scale
    assert np.max(np.abs(gy.cpu().numpy() - oy)) <= 1e-12 * scale


@pytest.mark.parametrize("n_ip,ions,pressure", [(3, 300, 1e-6), (1, 64, 3e-6)])
def test_beam_ion_turns_match_oracle(tmp_path, cuda_device, n_ip, ions, pressure):
    conf = small_conf(tmp_path, "beam_ion.conf", Np=500, filling="SINGLE10", xxCM_offset=0.3,
                      zzCM_offset=0.5)
    C = api.Config(conf)
    bi = C.beam_ion()
    bi.n_ip, bi.ions_per_passage, bi.pressure = n_ip, ions, pressure
    npb = np.full(C.nbunch, 500)
    ib = C.bunch_currents()
    beam = C.reference_beam(500)
    o = Oracle(C.params, C.bucket, npb, ib)
    t = api.Tracker(C.params, C.bucket, npb, ib)
    for i in range(C.nbunch):
        o.set_particles(i, beam[i])
        t.load_particles(i, beam[i])
    o.prepare()
    t.enable_beam_ion(bi)
    t.prepare()
    o.enable_beam_ion(bi)
    turns = 6
    so = o.run(turns)
    st = t.run(turns)
    assert stats_err(st, so).max() <= 1e-10
    co, ct = o.beam_ion_clouds(), t.beam_ion_clouds()
    assert co[:, 1:, 0].min() > 0
    for m in range(5):
        scale = np.abs(co[..., m]).max()
        assert np.max(np.abs(ct[..., m] - co[..., m])) <= 1e-11 * scale, m
    for i in range(C.nbunch):
        assert coord_err(t.get_particles(i), o.get_particles(i)).max() <= 1e-12, i
    # the ions moved the beam: same run without gas differs
    assert np.abs(co[..., 0]).max() > 0


def test_surrogate_stage_tracks_the_faddeeva_stage(tmp_path, cuda_device, trained_mlp):
    """The beam-ion stage with the learned field (trained with the standard
    settings on the project's own Faddeeva field) follows the Faddeeva
    stage: the audited relative field error |F_net - F| / |F| stays within
    the north star's 1e-4 at its maximum, the clouds and centroids agree to
    that level, the out-of-domain evaluations go to the Faddeeva field and
    no tensor-core wait fails."""
    mlp, _ = trained_mlp
    conf = small_conf(tmp_path, "beam_ion.conf", Np=2000, filling="SINGLE10", xxCM_offset=0.3, zzCM_offset=0.5)
    C = api.Config(conf)
    runs = {}
    for surr in (0, 1):
        bi = C.beam_ion()
        bi.n_ip, bi.ions_per_passage, bi.pressure, bi.surrogate, bi.audit_fraction = 4, 500, 1e-6, surr, 0.05
        t = api.Tracker(C.params, C.bucket, np.full(C.nbunch, 2000), C.bunch_currents())
        for i, b in enumerate(C.reference_beam(2000)):
            t.load_particles(i, b)
        t.enable_beam_ion(bi)
        if surr:
            t.use_mlp(mlp)
        t.prepare()
        runs[surr] = (t.run(8), t.beam_ion_clouds(), t.beam_ion_audit() if surr else None)
    (s0, c0, _), (s1, c1, audit) = runs[0], runs[1]
    n_audit, max_err, rms_err, fallbacks, failures = audit
    print("audit: %d evaluations, max %.2e, rms %.2e, %d fallbacks" % (n_audit, max_err, rms_err, fallbacks))
    assert failures == 0
    assert n_audit > 1000 and max_err <= 1e-4 and rms_err <= 1e-5, audit
    # centroids (relative to the rms size) and clouds agree to the field error
    assert stats_err(s1, s0).max() < 1e-5
    rel = np.abs(c1[..., 0] - c0[..., 0]).max() / np.abs(c0[..., 0]).max()
    assert rel < 1e-12      # ion counts do not depend on the field
    for m in (1, 2, 3, 4):
        assert np.abs(c1[..., m] - c0[..., m]).max() <= 1e-5 * np.abs(c0[..., 3:]).max(), m


def test_surrogate_growth_rate_within_one_percent(tmp_path, cuda_device, trained_mlp):
    """The vertical beam-ion instability grows at the same rate with the
    learned field as with the Faddeeva field (within 1 %): the 200-bunch
    train with 5e3 macroparticles per bunch, 4 interaction points at
    10 nTorr (growth within a few hundred turns), same beam, ions and
    seeds; the rate is fitted over the exponential rise of the rms bunch
    centroid (mbtrack_b200.analysis)."""
    from mbtrack_b200 import analysis
    mlp, _ = trained_mlp
    amp = {}
    for surr in (0, 1):
        C = api.Config(small_conf(tmp_path, "beam_ion.conf", Np=5000))
        bi = C.beam_ion()
        bi.n_ip, bi.pressure, bi.surrogate = 4, 10e-9, surr
        t = api.Tracker(C.params, C.bucket, np.full(C.nbunch, 5000), C.bunch_currents())
        t.generate_beam(3)
        t.enable_beam_ion(bi)
        if surr:
            t.use_mlp(mlp)
        t.prepare()
        amp[surr] = analysis.centroid_amplitude(t.run(450), "VER")
        if surr:
            a = t.beam_ion_audit()
            assert a[4] == 0 and a[1] <= 1e-4, a
        t.close()
    w = analysis.exponential_window(amp[0])
    assert w is not None and w[1] - w[0] >= 50, w
    k0, k1 = analysis.growth_rate(amp[0], w), analysis.growth_rate(amp[1], w)
    print("growth rate per turn: Faddeeva %.5e, learned %.5e (turns %d..%d)" % (k0, k1, w[0], w[1]))
    assert k0 > 0 and abs(k1 - k0) <= 0.01 * k0
