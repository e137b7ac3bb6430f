"""The product's C host (mbt_config_load / mbt_config_greens, a restatement
of input.c and transform_weak.c:288-471) against the parameters the
reference derived for the same files."""
import numpy as np
import pytest

from mbtrack_b200 import api
from mbtrack_b200.abi import params_to_dict
from tests.golden_cases import CASES, Case


@pytest.mark.parametrize("name", CASES)
def test_parser_matches_reference(name, tmp_path, libmbt):
    c = Case(name)
    cfg = api.Config(c.conf_file(tmp_path))
    got = params_to_dict(cfg.params)
    for k, v in c.params_dict.items():
        assert got[k] == v, "%s: %r != %r" % (k, got[k], v)
    assert np.array_equal(cfg.bucket, c.bucket)
    assert np.array_equal(cfg.bunch_currents(), c.ib)
    n = cfg.params.ncell
    assert np.array_equal(cfg.Gl[:n], c.Gl)
    assert np.array_equal(cfg.Gv[:n], c.Gv)
    assert np.array_equal(cfg.Gh[:n], c.Gh)


def test_baseline_configs_parse(libmbt):
    from tests.util import conf
    import os
    cwd = os.getcwd()
    try:
        os.chdir(os.path.dirname(os.path.dirname(conf("x"))) + "/..")
        for name, nb in (("single_bunch.conf", 1), ("uniform_fill.conf", 416), ("uneven_fill.conf", 321)):
            cfg = api.Config(conf(name))
            assert cfg.nbunch == nb
            assert cfg.params.nharm == 416
    finally:
        os.chdir(cwd)


def test_missing_key_is_an_error(tmp_path, libmbt):
    from tests.util import conf
    text = open(conf("single_bunch.conf")).read().replace("  Np = 100000\n", "")
    p = tmp_path / "bad.conf"
    p.write_text(text)
    with pytest.raises(api.MbtError) as e:
        api.Config(str(p))
    assert "Np" in str(e.value)


def test_duplicate_section_counts_as_missing(tmp_path, libmbt):
    # config_have_section (input.c:980-1006): a repeated section is not unique
    from tests.util import conf
    text = open(conf("single_bunch.conf")).read() + "\n[resonator_1]\n  Rs = 1\n"
    p = tmp_path / "dup.conf"
    p.write_text(text)
    cfg = api.Config(str(p))
    assert cfg.params.planeL == 0 and cfg.params.planeH == 0 and cfg.params.planeV == 0


def test_missing_chv_resets_chh(tmp_path, libmbt):
    # input.c:414-417: any missing coupling coefficient zeroes CHH
    from tests.util import conf
    text = open(conf("single_bunch.conf")).read().replace("  QV0 = 10.23\n", "  QV0 = 10.23\n  CHH = 5.0\n  CVV = 2.0\n")
    p = tmp_path / "chh.conf"
    p.write_text(text)
    cfg = api.Config(str(p))
    assert cfg.params.CHH == 0.0 and cfg.params.CVV == 2.0 and cfg.params.amp_dep_qv == 1


SCAN_CONFS = {
    "current": {"scan_type": 1, "Nscan": 3, "NrevScan": 8, "scan_start": 150.0, "scan_step": 30.0},
    "chroma": {"scan_type": 2, "Nscan": 2, "NrevScan": 5},
    "q_down": {"scan_type": 3, "Nscan": 4, "NrevScan": 6},
    "q_from": {"scan_type": 4, "Nscan": 3, "NrevScan": 7, "scan_start": 0.25},
}


def scan_conf(tmp_path, kind):
    from tests.util import add_section, small_conf
    path = small_conf(tmp_path, "uniform_fill.conf", filling="SINGLE10", NrevTot=1)
    return add_section(path, "scan", **SCAN_CONFS[kind])


def test_scan_setup(tmp_path, libmbt):
    """[scan] (input.c:807-846) and its set-up (input.c:1710-1736): NrevTot
    = Nscan x NrevScan, a current scan starts the ring at scan_start, Q
    scans divide or scale the longitudinal resonators' Q factors."""
    base = api.Config(small_conf_plain(tmp_path)).params
    cur = api.Config(scan_conf(tmp_path, "current")).params
    assert (cur.scan, cur.nscan, cur.nrev_scan, cur.nrev_tot) == (1, 3, 8, 24)
    assert cur.Iring == 150.0 and cur.scan_start == 150.0 and cur.scan_step == 30.0
    ch = api.Config(scan_conf(tmp_path, "chroma")).params
    assert (ch.scan, ch.nrev_tot, ch.scan_start, ch.Iring) == (2, 10, 0.0, base.Iring)
    qd = api.Config(scan_conf(tmp_path, "q_down")).params
    assert qd.scan_start == 0.25 and qd.scan_step == 0.25
    assert qd.lr_Q[0][0] == base.lr_Q[0][0] / 4
    qf = api.Config(scan_conf(tmp_path, "q_from")).params
    assert qf.scan_step == (1.0 - 0.25) / 2 and qf.lr_Q[0][0] == base.lr_Q[0][0] * 0.25


def small_conf_plain(tmp_path):
    from tests.util import small_conf
    return small_conf(tmp_path, "uniform_fill.conf", filling="SINGLE10", NrevTot=1)


@pytest.mark.parametrize("kind", sorted(SCAN_CONFS))
def test_scan_setup_matches_reference(tmp_path, kind, libmbt):
    """Every parameter after set-up equals the reference's for each scan type."""
    from oracle.binding import Reference, build_reference, reference_available
    if not reference_available() or build_reference() is None:
        pytest.skip("reference tree not present")
    conf = scan_conf(tmp_path, kind)
    ours = params_to_dict(api.Config(conf).params)
    ref = params_to_dict(Reference(conf, workdir=str(tmp_path)).params())
    for k in ("scan", "nscan", "nrev_scan", "scan_start", "scan_step", "nrev_tot", "Iring", "lr_Q"):
        assert ours[k] == ref[k], "%s: %r != %r" % (k, ours[k], ref[k])


def test_scan_rejects_bad_sections(tmp_path, libmbt):
    from tests.util import add_section, small_conf
    p = add_section(small_conf(tmp_path, "uniform_fill.conf", NrevTot=1), "scan", scan_type=7, Nscan=2, NrevScan=3)
    with pytest.raises(api.MbtError):
        api.Config(p)
    # a Q scan needs a longitudinal long-range resonator (input.c:1716-1720)
    d = tmp_path / "noq"
    d.mkdir()
    p = add_section(small_conf(d, "single_bunch.conf", NrevTot=1), "scan", scan_type=3, Nscan=2, NrevScan=3)
    with pytest.raises(api.MbtError):
        api.Config(p)


def _rw_first_bin(u):
    try:
        return (0,) + api.rw_first_bin(u)
    except api.MbtError:
        return (-1, 0.0, 0.0)


def test_rw_first_bin_against_reference_table(libmbt):
    """The reference interpolates a printed table (rw_table.c); its
    longitudinal entries carry a constant error of 4.6e-4 in the integral of
    the wake over the bin (the exact integral of the resistive-wall wake
    over all s is zero), so |ours - table| u stays below 4.7e-4; the
    transverse entries agree to 1.5e-4 relative.  Values from the
    reference's own functions (tests/golden/make_rw_golden.py)."""
    import os
    from tests.util import GOLDEN
    z = np.load(os.path.join(GOLDEN, "rw_first_bin.npz"))
    for u, lon_ref, trans_ref in zip(z["u"], z["lon"], z["trans"]):
        r, lon, trans = _rw_first_bin(u)
        assert r == 0
        assert abs(lon - lon_ref) * min(u, 2000.0) < 4.7e-4, u
        assert abs(trans / trans_ref - 1) < 1.5e-4, u
    assert _rw_first_bin(19.7)[0] == -1
    assert _rw_first_bin(2500.0)[1:] == _rw_first_bin(2000.0)[1:]


def test_rw_first_bin_is_the_bane_sands_bin_average(libmbt):
    """Independent check of the quadrature: the bin average of the
    Bane-Sands wake w(x) = e^-x cos(sqrt3 x)/3 - sqrt2/pi int t^2 e^(-t^2 x)
    / (t^6+8) dt, and of its running integral, by nested scipy quadrature
    of that definition."""
    from scipy.integrate import quad

    def w(x):
        inner = quad(lambda t: t * t * np.exp(-t * t * x) / (t ** 6 + 8), 0, np.inf, epsabs=1e-15, limit=200)[0]
        return np.exp(-x) * np.cos(np.sqrt(3) * x) / 3 - np.sqrt(2) / np.pi * inner

    for u in (25.0, 140.0):
        pts = [0, 0.5, 2, 6, 15, u]
        lon = sum(quad(w, a, b, epsabs=1e-14, limit=200)[0] for a, b in zip(pts[:-1], pts[1:])) / u
        # int_0^u W = int_0^u (u - x) w(x) dx
        trans = sum(quad(lambda x: (u - x) * w(x), a, b, epsabs=1e-13, limit=200)[0]
                    for a, b in zip(pts[:-1], pts[1:])) / u
        r, l2, t2 = _rw_first_bin(u)
        assert abs(l2 - lon) < 1e-9 * abs(lon) + 1e-13, (u, l2, lon)
        assert abs(t2 / trans - 1) < 1e-9, (u, t2, trans)


def test_rw_short_greens_match_reference(tmp_path, libmbt):
    """construct_greensfunc_RW (transform_weak.c:473-547) on top of the
    resonators: every bin from 1 on bit-identical to the reference's, bin 0
    apart by exactly the first-bin value difference times its factor."""
    from oracle.binding import Reference, build_reference, reference_available
    from tests.util import rw_short_conf
    if not reference_available() or build_reference() is None:
        pytest.skip("reference tree not present")
    conf = rw_short_conf(tmp_path)
    cfg = api.Config(conf)
    R = Reference(conf, workdir=str(tmp_path))
    R.prepare()
    Gl, Gv, Gh, _ = R.greens()
    p = cfg.params
    n = p.ncell
    assert (p.planeL, p.planeV, p.planeH) == (2, 2, 2)
    for ours, ref in ((cfg.Gl, Gl), (cfg.Gv, Gv), (cfg.Gh, Gh)):
        assert np.array_equal(ours[1:n], ref[1:n])
    import ctypes
    from oracle import binding
    tab = ctypes.CDLL(binding.REF_SO)
    Z0, c = 376.73, 2.997925e8
    binw = p.sigma_tau * p.dT * c
    for G, Gr, b, kind in ((cfg.Gl, Gl, p.beffL[1], 0), (cfg.Gv, Gv, p.beffV[1], 1), (cfg.Gh, Gh, p.beffH[1], 1)):
        s0 = (2 * b * b * p.rhorw / Z0) ** (1 / 3)
        u = binw / s0
        v = ctypes.c_double()
        f = tab.RW_table_LON if kind == 0 else tab.RW_table_TRANS
        f.argtypes = [ctypes.c_double, ctypes.POINTER(ctypes.c_double)]
        f(u, v)
        ours = _rw_first_bin(u)[1 + kind]
        fac = 4 * Z0 * c / (np.pi * b * b) * p.Lc if kind == 0 else 8 * Z0 * c / (np.pi * b ** 4) * s0 * p.Lc
        assert abs((G[0] - Gr[0]) - (ours - v.value) * fac) <= 1e-9 * abs(Gr[0]), kind


def test_rw_short_needs_wide_bins(tmp_path, libmbt):
    """input.c:1744-1756: bins narrower than 20 s0 are refused (the
    reference prints the error and runs on with a half-built set-up)."""
    from tests.util import rw_short_conf
    with pytest.raises(api.MbtError) as e:
        api.Config(rw_short_conf(tmp_path, Nsigma=0.5))
    assert "binwidth" in str(e.value)
