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
