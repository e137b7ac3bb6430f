"""Parity of the CUDA path (libmbt through its C-ABI) with the oracle.

Bars: coordinates within 1e-12 relative after N turns (relative to each
coordinate's rms spread); centroid and rms histories within 1e-10 (the rms
relative to itself, the centroids relative to the plane's rms and, as
tests.util.centroid_err, relative to the centroid history's own size);
histogram counts bit-exact on identical coordinates."""
import numpy as np
import pytest

from mbtrack_b200 import api
from mbtrack_b200.abi import MBT_NOISE_INJECTED
from oracle.binding import Oracle
from tests.golden_cases import CASES, Case
from tests.util import centroid_err, coord_err, small_conf, stats_err

pytestmark = pytest.mark.gpu

COORD_TOL = 1e-12
STATS_TOL = 1e-10


def tracker_for(c, noise=None):
    mode = MBT_NOISE_INJECTED if c.params.quantum else 0
    return api.Tracker(c.params, c.bucket, c.np, c.ib, c.Gl, c.Gv, c.Gh, noise=mode)


@pytest.mark.parametrize("name", CASES)
def test_fixture_cases(name, cuda_device, libmbt):
    c = Case(name)
    t = tracker_for(c)
    init = c.bunch_slices(c.init)
    for i in range(c.nb):
        t.load_particles(i, init[i])
    st0 = t.prepare()
    assert np.max(stats_err(st0, c.init_stats)) < STATS_TOL
    if c.params.quantum:
        t.set_deviates(c.deviates, c.turns)
    st = t.run(c.turns)
    assert np.max(stats_err(st, c.stats)) < STATS_TOL
    assert np.max(centroid_err(st, c.stats)) < STATS_TOL, np.max(centroid_err(st, c.stats))
    final = c.bunch_slices(c.final)
    worst = 0.0
    for i in range(c.nb):
        worst = max(worst, np.max(coord_err(t.get_particles(i), final[i])))
    assert worst < COORD_TOL, worst
    s = t.state()
    assert abs(s.Vrf0 - c.vrf_phi[0]) <= 1e-12 * abs(c.vrf_phi[0])
    assert abs(s.phai0 - c.vrf_phi[1]) <= 1e-12 * abs(c.vrf_phi[1])
    t.close()


def _oracle_and_tracker(cfg, noise_injected=False):
    o = Oracle(cfg.params, cfg.bucket, np.full(cfg.nbunch, cfg.params.np_model),
               cfg.bunch_currents(), cfg.Gl, cfg.Gv, cfg.Gh)
    o.generate_beam()
    t = api.Tracker.from_config(cfg, noise=MBT_NOISE_INJECTED if noise_injected else 0)
    for i in range(cfg.nbunch):
        t.load_particles(i, o.get_particles(i))
    return o, t


@pytest.mark.parametrize("scan", [
    {"scan_type": 1, "Nscan": 3, "NrevScan": 25, "scan_start": 120.0, "scan_step": 40.0},
    {"scan_type": 4, "Nscan": 3, "NrevScan": 25, "scan_start": 0.5},
])
def test_scan_steps(tmp_path, scan, cuda_device, libmbt):
    """Current scan (bucket and bunch currents, factG and the weighting of
    the resistive-wall history change at each boundary) and Q scan (only the
    resistive-wall trigger count restarts, here after 25 of its 50 kicks),
    run in calls whose ends fall inside and on the scan intervals."""
    from tests.util import add_section, add_tracking_keys
    path = small_conf(tmp_path, "uniform_fill.conf", Np=300, Nmlt=3, filling="SINGLE20", xxCM_offset=0.05,
                      EnableQuantum=0, NrevTot=1)
    add_tracking_keys(path, triggerRW=1)
    cfg = api.Config(add_section(path, "scan", **scan))
    assert cfg.params.nrev_tot == 75
    o, t = _oracle_and_tracker(cfg)
    so0, st0 = o.prepare(), t.prepare()
    assert np.max(stats_err(st0, so0)) < STATS_TOL
    for n in (7, 18, 30, 20):
        so = o.run(n)
        st = t.run(n)
        assert np.max(stats_err(st, so)) < STATS_TOL, n
        worst = max(np.max(coord_err(t.get_particles(i), o.get_particles(i))) for i in range(cfg.nbunch))
        assert worst < COORD_TOL, (n, worst)
    t.close()


def test_short_range_rw(tmp_path, cuda_device, libmbt):
    """Short-range resistive wall in three planes (its Green's functions
    from mbt_config_greens) with the broadband resonators, 300 turns."""
    from tests.util import rw_short_conf
    cfg = api.Config(rw_short_conf(tmp_path, Np=20000, xxCM_offset=0.05, zzCM_offset=0.02))
    assert (cfg.params.planeL, cfg.params.planeV, cfg.params.planeH) == (2, 2, 2)
    o, t = _oracle_and_tracker(cfg)
    so0, st0 = o.prepare(), t.prepare()
    assert np.max(stats_err(st0, so0)) < STATS_TOL
    so, st = o.run(300), t.run(300)
    assert np.max(stats_err(st, so)) < STATS_TOL
    assert np.max(coord_err(t.get_particles(0), o.get_particles(0))) < COORD_TOL
    t.close()


def test_ragged_and_tiny_bunches(tmp_path, cuda_device, libmbt):
    """Ten bunches of 1 .. 20000 macroparticles (sizes that do not fill a
    warp, a 512-particle stage or a tile; 8193 and 20000 span several
    tiles), resistive wall and the HOM, one bunch displaced by 7 sigma in
    time so that part of it falls outside the binning window (the
    out-of-range counters): 25 turns against the oracle."""
    from tests.util import small_conf as sc
    cfg = api.Config(sc(tmp_path, "uniform_fill.conf", filling="SINGLE10", Nmlt=3, EnableQuantum=0,
                        xxCM_offset=0.05, zzCM_offset=0.02))
    np_ = np.array([1, 2, 31, 33, 511, 513, 1025, 4097, 8193, 20000], dtype=np.int32)
    assert cfg.nbunch == len(np_)
    o = Oracle(cfg.params, cfg.bucket, np_, cfg.bunch_currents(), cfg.Gl, cfg.Gv, cfg.Gh)
    o.generate_beam()
    X = o.get_particles(6).reshape(6, -1).copy()
    X[0] += 7.0 * cfg.params.sigma_tau
    o.set_particles(6, X.ravel())
    t = api.Tracker(cfg.params, cfg.bucket, np_, cfg.bunch_currents(), cfg.Gl, cfg.Gv, cfg.Gh)
    for i in range(cfg.nbunch):
        t.load_particles(i, o.get_particles(i))
    so0, st0 = o.prepare(), t.prepare()
    so, st = o.run(25), t.run(25)
    many = np_ >= 2                                  # one macroparticle has no rms to scale by
    assert np.max(stats_err(st0[many], so0[many])) < STATS_TOL
    assert np.max(stats_err(st[:, many], so[:, many])) < STATS_TOL
    assert np.max(np.abs(st[:, 0, :3] - so[:, 0, :3])) <= 1e-12 * np.max(np.abs(so[:, 0, :3]))
    worst = max(np.max(coord_err(t.get_particles(i), o.get_particles(i))) for i in range(cfg.nbunch))
    assert worst < COORD_TOL, worst
    assert t.state().n_trash_high + t.state().n_trash_low > 0
    t.close()


def test_whole_beam_transfers_on_ragged_bunches(tmp_path, cuda_device, libmbt):
    """mbt_load_all / mbt_get_all (one copy each way and a layout kernel) on
    bunches of 1 .. 20000 macroparticles: the beam comes back bit for bit,
    and after some turns with the resistive wall (a pending kick in the
    slopes) it equals the per-bunch exports."""
    from tests.util import small_conf as sc
    cfg = api.Config(sc(tmp_path, "uniform_fill.conf", filling="SINGLE10", Nmlt=3, EnableQuantum=0))
    np_ = np.array([1, 2, 31, 33, 511, 513, 1025, 4097, 8193, 20000], dtype=np.int32)
    t = api.Tracker(cfg.params, cfg.bucket, np_, cfg.bunch_currents(), cfg.Gl, cfg.Gv, cfg.Gh)
    buf = np.random.default_rng(4).normal(0, 1e-3, 6 * int(np_.sum()))
    t.load_all(buf)
    assert np.array_equal(t.get_all(), buf)
    per = [t.get_particles(i) for i in range(cfg.nbunch)]
    assert np.array_equal(np.concatenate([x.ravel() for x in per]), buf)
    t.prepare()
    t.run(4, stats=False)
    got = t.get_all()
    per = np.concatenate([t.get_particles(i).ravel() for i in range(cfg.nbunch)])
    assert np.array_equal(got, per)
    t.close()


def test_single_bunch_full_size_2000_turns(tmp_path, cuda_device, libmbt):
    """Single bunch, 1e5 macroparticles, broadband resonator in three planes,
    noise off, 2000 turns: checked after 1, 10 and 2000 turns."""
    cfg = api.Config(small_conf(tmp_path, "single_bunch.conf", xxCM_offset=0.05, zzCM_offset=0.02))
    o, t = _oracle_and_tracker(cfg)
    so0, st0 = o.prepare(), t.prepare()
    assert np.max(stats_err(st0, so0)) < STATS_TOL
    done = 0
    for upto in (1, 10, 2000):
        n = upto - done
        so = o.run(n)
        st = t.run(n)
        done = upto
        assert np.max(stats_err(st, so)) < STATS_TOL, upto
        assert np.max(centroid_err(st, so)) < STATS_TOL, (upto, centroid_err(st, so))
        err = coord_err(t.get_particles(0), o.get_particles(0))
        assert np.max(err) < COORD_TOL, (upto, err)


def test_uniform_fill_all_buckets_with_noise(tmp_path, cuda_device, libmbt):
    """All 416 buckets, RW over a 50-turn history plus the HOM, injected
    deviates (reduced macroparticle count so the oracle stays fast), 64
    turns: past the first wrap of the (Nmlt + 2) h = 52 x 416 slot history
    of the bunch dipoles (worker_weakweak.c:206, transform_weak.c:813-824)."""
    cfg = api.Config(small_conf(tmp_path, "uniform_fill.conf", Np=64, xxCM_offset=0.05))
    assert cfg.params.Nmlt == 50 and cfg.nbunch == 416
    o, t = _oracle_and_tracker(cfg, noise_injected=True)
    o.prepare()
    t.prepare()
    turns = 64
    so, dev = o.run(turns, record=True)
    t.set_deviates(dev, turns)
    st = t.run(turns)
    assert np.max(stats_err(st, so)) < STATS_TOL
    assert np.max(centroid_err(st, so)) < STATS_TOL, np.max(centroid_err(st, so))
    worst = max(np.max(coord_err(t.get_particles(i), o.get_particles(i))) for i in range(cfg.nbunch))
    assert worst < COORD_TOL


def test_uneven_fill_feedback(tmp_path, cuda_device, libmbt):
    """Uneven fill with the camshaft, RF feedback on the detuned fundamental
    cavity (averaging loop, feedback_rf.c:5-34, worker_weakweak.c:268-278),
    RW over 50 turns and the HOM, 64 turns: the feedback samples, the
    phasors and the dipole history all run through their long memories."""
    cfg = api.Config(small_conf(tmp_path, "uneven_fill.conf", Np=32, EnableQuantum=0))
    o, t = _oracle_and_tracker(cfg)
    so0, st0 = o.prepare(), t.prepare()
    assert np.max(stats_err(st0, so0)) < STATS_TOL
    so = o.run(64)
    st = t.run(64)
    assert np.max(stats_err(st, so)) < STATS_TOL
    assert np.max(centroid_err(st, so)) < STATS_TOL, np.max(centroid_err(st, so))
    v, _ = o.state(0)
    s = t.state()
    assert abs(s.Vrf0 - v[0]) < 1e-11 * abs(v[0]) and abs(s.phai0 - v[1]) < 1e-11 * abs(v[1])


def test_histogram_counts_bit_exact(tmp_path, cuda_device, libmbt):
    """On identical coordinates the device binning (clamped and dropped
    histograms, transform_weak.c:608-631 and :839-865) equals the oracle's:
    counts bit for bit, position sums to rounding."""
    c = Case("feedback_hc")
    o = Oracle(c.params, c.bucket, c.np, c.ib, c.Gl, c.Gv, c.Gh)
    o.generate_beam()
    o.prepare()
    o.run(7)
    X = [o.get_particles(i) for i in range(c.nb)]
    t = tracker_for(c)
    for i in range(c.nb):
        t.load_particles(i, X[i])
    t.prepare()
    o2 = Oracle(c.params, c.bucket, c.np, c.ib, c.Gl, c.Gv, c.Gh)
    for i in range(c.nb):
        o2.set_particles(i, X[i])
    o2.prepare()                                   # dropped histograms of X
    dropped = [o2.histograms(i)[3:5] for i in range(c.nb)]
    o2.run(1)                                      # clamped histograms of X
    for i in range(c.nb):
        g = t.histograms(i)
        r = o2.histograms(i)
        assert np.array_equal(g[0], r[0]), "clamped counts, bunch %d" % i
        assert np.array_equal(g[3], dropped[i][0]), "dropped counts, bunch %d" % i
        scale = np.max(np.abs(X[i][1])) * c.np[i]
        assert np.max(np.abs(g[2] - r[2])) <= 1e-13 * scale
        assert np.max(np.abs(g[4] - dropped[i][1])) <= 1e-13 * scale


def test_track_call_matches_resident_run(tmp_path, cuda_device, libmbt):
    """mbt_track (host buffers in and out) gives the device-resident result."""
    c = Case("train_rw_hom")
    a = tracker_for(c)
    b = tracker_for(c)
    init = c.bunch_slices(c.init)
    for i in range(c.nb):
        a.load_particles(i, init[i])
    a.prepare()
    sa = a.run(5)
    buf = np.concatenate([x.ravel() for x in init])
    sb = np.zeros_like(sa)
    b.track(buf, 5, sb)
    assert np.array_equal(sa, sb)
    assert np.array_equal(a.get_all(), buf)


def test_errors_are_reported(cuda_device, libmbt):
    c = Case("single_noiseoff")
    t = tracker_for(c)
    with pytest.raises(api.MbtError) as e:
        t.run(1)
    assert e.value.code == -5
    with pytest.raises(api.MbtError) as e:
        t.load_particles(0, np.zeros(6 * 3))
    assert e.value.code == -1


def test_amplitude_invariants(cuda_device, libmbt):
    """ampinv / ampinv_cm (statistics.c:163-195) of every turn, from the
    device moments, against the oracle after the same turns."""
    c = Case("single_noiseoff")
    t = tracker_for(c)
    init = c.bunch_slices(c.init)
    t.load_particles(0, init[0])
    t.prepare()
    o = Oracle(c.params, c.bucket, c.np, c.ib, c.Gl, c.Gv, c.Gh)
    o.set_particles(0, init[0])
    o.prepare()
    for turns in (1, 9):
        st, ai = t.run_ampinv(turns)
        o.run(turns)
        ref = o.ampinv(0)
        got = ai[-1, 0]
        for k in (1, 2):                       # HOR, VER (LON Twiss are 0 in the reference)
            assert abs(got[k] - ref[k]) <= 1e-10 * abs(ref[k])
            assert abs(got[3 + k] - ref[3 + k]) <= 1e-10 * abs(ref[k])
        assert got[0] == 0.0 and got[3] == 0.0


def test_tile_sizes_do_not_change_the_physics(tmp_path, cuda_device):
    """Re-tiling (mbt_set_tiles, as the autotuner does) changes only the
    grouping of the moment sums: statistics agree to rounding, counts are
    exact; the autotuner returns valid sizes."""
    conf = small_conf(tmp_path, "uneven_fill.conf", Np=4000)
    C = api.Config(conf)
    rng = np.random.default_rng(3)
    npb = rng.integers(1000, 40000, C.nbunch).astype(np.int32)
    beams = None
    out = []
    for tiles in ([4096, 4096, 4096], [512, 2048, 8192]):
        t = api.Tracker(C.params, C.bucket, npb, C.bunch_currents(), C.Gl, C.Gv, C.Gh, seed=5)
        if beams is None:
            t.generate_beam(9)
            beams = [t.get_particles(i) for i in range(C.nbunch)]
        else:
            for i, b in enumerate(beams):
                t.load_particles(i, b)
        t.prepare()
        t.set_tiles(tiles)
        out.append((t.run(10), t.histograms(7)[0]))
        if tiles[0] == 512:
            chosen = t.autotune(trial_turns=2)
            assert all(512 <= x <= 8192 and (x & (x - 1)) == 0 for x in chosen)
    from tests.util import stats_err
    assert stats_err(out[1][0], out[0][0]).max() < 1e-11
    assert np.array_equal(out[1][1], out[0][1])


def test_plain_and_general_particle_maps_agree(tmp_path, cuda_device, libmbt):
    """The particle pass compiles the map twice: for the common ring (all
    planes tracked, no harmonic cavity, no amplitude detuning, no dispersion
    at the kick point), chosen per launch, and in its general form.  The same
    ring with one active harmonic cavity of zero voltage runs the general
    form; with the same beam and the same Philox noise both give the same
    turns to the parity tolerances (the two forms round alike but the
    compiler may contract their multiply-adds differently)."""
    runs = []
    for i, extra in enumerate(("", "\n[active_HC_1]\n  Vpeak = 0.0\n  nHC = 3.0\n  phi_aHC = 0.0\n")):
        d = tmp_path / ("run%d" % i)
        d.mkdir()
        path = small_conf(d, "single_bunch.conf", Np=4096, EnableQuantum=1, xxCM_offset=0.05, zzCM_offset=0.02)
        with open(path, "a") as f:
            f.write(extra)
        cfg = api.Config(path)
        assert cfg.params.n_active_hc == i
        t = api.Tracker.from_config(cfg, seed=4321)
        t.generate_beam(11)
        t.prepare()
        st = t.run(40)
        runs.append((st, t.get_particles(0)))
        t.close()
    (sa, pa), (sb, pb) = runs
    assert np.max(stats_err(sb, sa)) < STATS_TOL
    assert np.max(centroid_err(sb, sa)) < STATS_TOL
    assert np.max(coord_err(pb, pa)) < COORD_TOL
