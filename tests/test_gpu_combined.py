"""The combined configuration (uneven fill with the camshaft bunch,
resistive wall over 50 turns, HOM, RF feedback with its generator loop,
per-macroparticle beam-ion with the learned field and its audit), reduced
so that the oracle can follow it: macroparticles proportional to the bunch
charge (20 .. 200), 4 interaction points, 20 macro-ions per passage at
1000x the pressure, 12 turns.

The Faddeeva-field run matches the oracle's restatement (statistics 1e-10,
coordinates 1e-12 of their spread); the learned-field run follows it within
the audited field error; the reference's output files, the bunch-by-bunch
centroid histories among them, are written for every turn."""
import os

import numpy as np
import pytest

from mbtrack_b200 import api
from oracle.binding import Oracle
from tests.util import centroid_err, coord_err, small_conf, stats_err

pytestmark = pytest.mark.gpu

TURNS = 12


def _np_by_charge(frac, lo, hi, total):
    k0, k1 = 1e-6, 1e15
    for _ in range(200):
        k = np.sqrt(k0 * k1)
        if np.clip(np.rint(k * frac), lo, hi).sum() < total:
            k0 = k
        else:
            k1 = k
    return np.clip(np.rint(np.sqrt(k0 * k1) * frac), lo, hi).astype(np.int32)


def test_combined_configuration(tmp_path, cuda_device, trained_mlp):
    mlp, _ = trained_mlp
    conf = small_conf(tmp_path, "combined.conf", NrevTot=TURNS, NrevMon=1, EnableQuantum=0, xxCM_offset=0.2,
                      zzCM_offset=0.3)
    C = api.Config(conf)
    assert C.nbunch == 321 and C.params.rffb and C.params.rffb_gain == 10.0 and C.params.rffb_delay == 1
    npb = _np_by_charge(np.asarray(C.ib_frac), 20, 200, 30000)
    assert npb.min() >= 20 and npb.max() == 200 and len(set(npb.tolist())) > 50
    ib = C.bunch_currents()

    def beam_ion(surr):
        bi = C.beam_ion()
        bi.n_ip, bi.ions_per_passage, bi.pressure, bi.surrogate, bi.audit_fraction = 4, 20, 1e-6, surr, 0.05
        return bi

    o = Oracle(C.params, C.bucket, npb, ib, C.Gl, C.Gv, C.Gh)
    o.generate_beam()
    beam = [o.get_particles(i) for i in range(C.nbunch)]
    runs = {}
    for surr in (0, 1):
        t = api.Tracker(C.params, C.bucket, npb, ib, C.Gl, C.Gv, C.Gh)
        for i, b in enumerate(beam):
            t.load_particles(i, b)
        t.enable_beam_ion(beam_ion(surr))
        if surr:
            t.use_mlp(mlp)
        st0 = t.prepare()
        if surr:
            work = str(tmp_path / "work")
            os.makedirs(work)
            ocfg, bunch_out = C.output()
            w = api.Writer(work, C.params, ocfg, bunch_out, C.bucket, ib)
            w.wakes(C.Gl, C.Gv, C.Gh)
            w.begin(st0)
        st, ai = t.run_ampinv(TURNS)
        if surr:
            w.turns(st, ai)
            w.end(t.get_stats())
            w.close()
        runs[surr] = (st, [t.get_particles(i) for i in range(C.nbunch)], t.beam_ion_audit() if surr else None,
                      t.state())
        t.close()
    o.prepare()
    o.enable_beam_ion(beam_ion(0))
    so = o.run(TURNS)
    (s0, x0, _, state0), (s1, x1, audit, _) = runs[0], runs[1]
    # Faddeeva-field run against the oracle
    assert np.max(stats_err(s0, so)) < 1e-10
    assert np.max(centroid_err(s0, so)) < 1e-10
    assert max(np.max(coord_err(x0[i], o.get_particles(i))) for i in range(C.nbunch)) < 1e-12
    v, _ = o.state(0)
    assert abs(state0.Vrf0 - v[0]) < 1e-11 * abs(v[0]) and abs(state0.phai0 - v[1]) < 1e-11 * abs(v[1])
    # learned-field run: audited error within the bar, statistics close
    n_audit, max_err, rms_err, fallbacks, failures = audit
    print("audit: %d evaluations, max %.2e, rms %.2e, %d fallbacks" % (n_audit, max_err, rms_err, fallbacks))
    assert failures == 0 and n_audit > 0 and max_err <= 1e-4
    # at 1000x the pressure the ions drive the bunches hard: the field
    # differences (a few 1e-6) grow over the turns, to 1e-5 of the rms here
    assert np.max(stats_err(s1, s0)) < 1e-4
    # the reference's files: bunch-by-bunch centroids of every turn
    for plane in ("LON", "HOR", "VER"):
        rows = [l.split() for l in open(os.path.join(work, "bunchbybunch_%s.dat" % plane)) if not l.startswith("#")]
        assert len(rows) == TURNS and all(len(r) == 2 + C.nbunch for r in rows), plane
        col = {"LON": 0, "HOR": 1, "VER": 2}[plane]
        got = np.array([[float(x) for x in r[2:]] for r in rows])
        assert np.allclose(got, s1[:, :, col], rtol=1e-7, atol=0), plane
