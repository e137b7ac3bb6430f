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
