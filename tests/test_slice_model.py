"""Slice model (BunchModel = STRONG) with fast beam-ion interaction, on the
CPU: the oracle (oracle/ws_oracle.c) against the reference's own functions
(live through oracle/ref_ws_harness.c, and through the golden fixtures
tests/golden/make_slice_golden.py made from them), and the product's host
side of libmbt -- configuration reader and slicing -- against the
reference's set-up (mbtrack-mpi.c:61-81, bunch_strong.c:59-198)."""
import os

import numpy as np
import pytest

from mbtrack_b200 import api
from oracle import binding
from tests.util import GOLDEN, SLICE_CASES, SLICE_TURNS, SLICE_UNEVEN, SLICE_UNEVEN_TURNS, slice_conf

DERIVED = ("nslc", "fbii", "np", "ngrid", "ndivs", "sgm_xx", "sgm_zz", "sgmatau", "max_tau", "dtau", "agLOCx",
           "agLOCz", "agABSx", "agABSz", "deltT", "factBE", "factF", "Ldmsgm", "Gamma", "kick_factor")
BASE = ("nharm", "E0", "T0", "wrf", "Vrf0", "phai0", "Urad", "ac", "QH0", "QV0", "Lc", "Iring", "Nmlt",
        "triggerRW", "rw_long", "nrev_tot", "nrev_mon")


def _golden(case):
    return np.load(os.path.join(GOLDEN, "slice_fbii_%s.npz" % case))


def _product(tmp_path, case, **over):
    """mbt_ws_params, buckets and currents [mA] from the product's reader."""
    w, bucket, frac = api.SliceModel.config(slice_conf(tmp_path, case, **over))
    L = api.lib()
    ib = np.array([L.mbt_bunch_current(w.base, len(bucket), float(f)) * 1e3 for f in frac])
    return w, bucket, ib


def _same(a, b):
    return np.array_equal(a, b, equal_nan=True)


@pytest.mark.parametrize("case", sorted(SLICE_CASES))
def test_oracle_matches_golden(tmp_path, libmbt, case):
    """The oracle reproduces the reference's slice model bit for bit: the
    slicing of the reference's particles, 30 turns of slice centroids, ion
    centroids, bunch zz means, monitor statistics and the final slices."""
    g = _golden(case)
    w, bucket, ib = _product(tmp_path, case)
    assert np.array_equal(bucket, g["bucket"]) and _same(ib, g["ibunch"])
    npop, nofe, _ = binding.slice_beam(w, g["particles"])
    assert np.array_equal(npop, g["npop"]) and np.array_equal(nofe, g["nofe"])
    o = binding.OracleSlices(w, bucket, ib, npop, nofe)
    o.set_slices(g["slices0"])
    cm, ion, zcm, st = o.run(SLICE_TURNS)
    for name, got in (("cm", cm), ("ion", ion), ("zcm", zcm), ("stats", st)):
        assert _same(got, g[name]), name
    assert _same(o.slices_state(), g["slices"])
    # the dynamics are live: ions pull the slices, the bunches move
    assert np.isfinite(ion[:, 1:]).all() and np.abs(ion[:, 1:]).max() > 0
    assert np.abs(np.diff(cm[:, :, 4], axis=0)).max() > 0


@pytest.mark.parametrize("case", sorted(SLICE_CASES))
def test_product_slicing_matches_reference(tmp_path, libmbt, case):
    """mbt_ws_slice_beam (host C of libmbt) slices the reference's particles
    as strong_generate_eCMs does: populations and local-grid counts equal
    to the reference's, slice centroids equal to the oracle's
    restatement."""
    g = _golden(case)
    w, _, _ = _product(tmp_path, case)
    p = g["particles"]
    npop, nofe, cm4 = api.SliceModel.slice_beam(w, p)
    assert np.array_equal(npop, g["npop"]) and np.array_equal(nofe, g["nofe"])
    onpop, onofe, ocm4 = binding.slice_beam(w, p)
    assert np.array_equal(npop, onpop) and np.array_equal(nofe, onofe) and _same(cm4, ocm4)
    # particles beyond the window land in the overflow cell, not in a slice
    far = p.copy()
    far[0, :10] = -50 * w.sgmatau
    npop2, _, _ = api.SliceModel.slice_beam(w, far)
    assert npop2.sum() == npop.sum() - np.count_nonzero(
        np.minimum(((7.0 - p[0, :10] / w.sgmatau) / 0.3).astype(int), w.slices) < w.slices)


@pytest.mark.reference
@pytest.mark.parametrize("case", sorted(SLICE_CASES))
def test_config_matches_reference(tmp_path, libmbt, case):
    """mbt_ws_config_load gives the reference's set-up values: grid, slice
    duration, field and ion constants, ring and tracking fields."""
    if not binding.reference_available() and not os.path.exists(binding.REF_SO):
        pytest.skip("reference harness unavailable")
    path = slice_conf(tmp_path, case)
    r = binding.ReferenceSlices(path)
    want = r.params()
    w, bucket, ib = _product(tmp_path, case)
    for f in DERIVED:
        assert getattr(w, f) == getattr(want, f), f
    for f in BASE:
        assert getattr(w.base, f) == getattr(want.base, f), f
    for f in ("alpha1", "beta1", "gamma1", "track_plane"):
        assert list(getattr(w.base, f)) == list(getattr(want.base, f)), f
    assert w.base.beffH[0] == want.base.beffH[0] and w.base.beffV[0] == want.base.beffV[0]
    assert np.array_equal(bucket, r.bucket) and _same(ib, r.ibunch)


@pytest.mark.reference
@pytest.mark.parametrize("over", [{"EnableFBII": 0}, {"EnableRW_long": 0}, {"Nslc": 3}, {"NrevMon": 1}],
                         ids=["no_fbii", "no_rw", "nslc3", "mon_every_turn"])
def test_oracle_matches_reference_live(tmp_path, libmbt, over):
    """Variants run side by side with the reference's functions, bit for
    bit: beam-ion off (resistive wall only), resistive wall off, the
    reference's default Nslc = 3 (all particles fall in its overflow cell:
    empty slices, no ions), statistics every turn."""
    if not binding.reference_available() and not os.path.exists(binding.REF_SO):
        pytest.skip("reference harness unavailable")
    path = slice_conf(tmp_path, "train", **over)
    r = binding.ReferenceSlices(path)
    w, bucket, ib = _product(tmp_path, "train", **over)
    o = binding.OracleSlices(w, bucket, ib, r.npop, r.nofe)
    o.set_slices(r.slices_state())
    n = 15
    a = r.run(n, w.base.nrev_mon)
    b = o.run(n)
    for name, x, y in zip(("cm", "ion", "zcm", "stats"), a, b):
        assert _same(x, y), name
    assert _same(r.slices_state(), o.slices_state())
    for ib_ in (0, len(bucket) - 1):
        e1, i1 = r.bunch_fields(ib_)
        e2, i2 = o.bunch_fields(ib_)
        if w.fbii:
            assert _same(e1, e2) and _same(i1, i2)


@pytest.mark.reference
def test_interpolation_matches_reference(tmp_path, libmbt):
    """The grid interpolation (get_linearly_interpolated_Efields) of the
    oracle equals the reference's at points inside, on the edges of and far
    outside the 5 x 5 grid, both signs of each axis."""
    if not binding.reference_available() and not os.path.exists(binding.REF_SO):
        pytest.skip("reference harness unavailable")
    path = slice_conf(tmp_path, "train")
    r = binding.ReferenceSlices(path)
    r.run(2, 10)
    w, bucket, ib = _product(tmp_path, "train")
    o = binding.OracleSlices(w, bucket, ib, r.npop, r.nofe)
    o.set_slices(r.slices_state())
    r.set_slices(r.slices_state())
    r.run(1, 10)
    o.run(1)
    rng = np.random.default_rng(5)
    ax, az = w.agABSx, w.agABSz
    x = np.concatenate([rng.uniform(-4, 4, 400) * ax, np.arange(-3, 4) * ax, rng.uniform(-60, 60, 100) * ax,
                        [0.0, -0.0, 2.5 * ax, -2.5 * ax]])
    y = np.concatenate([rng.uniform(-4, 4, 400) * az, np.arange(-3, 4) * az, rng.uniform(-60, 60, 100) * az,
                        [0.0, -0.0, -2.5 * az, 2.5 * az]])
    for icell in (0, 20, 23, 40):
        assert _same(r.interp(3, icell, x, y), o.interp(3, icell, x, y))


def test_config_refusals(tmp_path, libmbt):
    """The slice-model reader refuses what the model cannot run: more than
    49 slices, a beam no flatter than round, a weak-model file; and the
    weak-model reader refuses a slice-model file."""
    with pytest.raises(api.MbtError, match="Nslc"):
        api.SliceModel.config(slice_conf(tmp_path, "train", Nslc=25))
    with pytest.raises(api.MbtError, match="sgm_zz"):
        api.SliceModel.config(slice_conf(tmp_path, "train", sgm_zz=0.3))
    with pytest.raises(api.MbtError, match="STRONG"):
        api.SliceModel.config(os.path.join(os.path.dirname(os.path.abspath(__file__)), "confs",
                                           "uniform_fill.conf"))
    with pytest.raises(api.MbtError, match="STRONG"):
        api.Config(slice_conf(tmp_path, "train"))


def test_slice_model_needs_a_device(tmp_path, libmbt):
    """Without a GPU the device context is refused with an error code (no
    CPU fallback)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    w, bucket, ib = _product(tmp_path, "train")
    S = w.slices
    with pytest.raises(api.MbtError) as e:
        api.SliceModel(w, bucket, ib, np.ones(S, np.int32), np.zeros((S, 5, 5), np.int32))
    assert e.value.code == -7


@pytest.mark.reference
@pytest.mark.parametrize("case", ["train", "nofbii"])
def test_writer_matches_reference_files(tmp_path, libmbt, case):
    """mbt_ws_writer_* writes the slice-model manager's files byte for byte
    as the reference's own writers do on the same numbers: CMmotionsV.out,
    CMImotionsH/V.out, ampinv_<P>_<turn>.dat every NrevMon (with the
    reference's history indexing), ampinv/cmpos means, gendst files."""
    if not binding.reference_available() and not os.path.exists(binding.REF_SO):
        pytest.skip("reference harness unavailable")
    over = {"NrevTot": 30, "NrevMon": 10}
    if case == "nofbii":
        over["EnableFBII"] = 0
    for pl in ("LON", "HOR", "VER"):
        over["gendst_datafile_" + pl] = str(tmp_path / ("ref_gendst_" + pl))
    path = slice_conf(tmp_path, "train", **over)
    ref_dir, mine_dir = tmp_path / "ref", tmp_path / "mine"
    ref_dir.mkdir()
    mine_dir.mkdir()
    r = binding.ReferenceSlices(path, workdir=str(ref_dir))
    r.files(True)
    r.write_distribution()
    cm, ion, zcm, st = r.run(30, 10)
    r.finish()
    w, bucket, _ = _product(tmp_path, "train", **over)
    wr = api.SliceWriter(str(mine_dir), w, bucket)
    wr.turns(ion[:13], zcm[:13], st[:2])
    wr.turns(ion[13:], zcm[13:], st[2:])
    soa, _ = api.SliceModel.reference_beam(w, len(bucket))
    mine_g = [str(tmp_path / ("mine_gendst_" + pl)) for pl in ("LON", "HOR", "VER")]
    wr.distribution(mine_g, soa)
    wr.close()
    names = sorted(os.listdir(ref_dir))
    assert names == sorted(os.listdir(mine_dir))
    assert ("CMImotionsH.out" in names) == (case == "train") and "ampinv_VER_21.dat" in names
    for n in names:
        assert (ref_dir / n).read_bytes() == (mine_dir / n).read_bytes(), n
    for pl, m in zip(("LON", "HOR", "VER"), mine_g):
        assert (tmp_path / ("ref_gendst_" + pl)).read_bytes() == open(m, "rb").read(), pl


@pytest.mark.parametrize("case", sorted(SLICE_CASES))
def test_reference_beam_matches_reference(tmp_path, libmbt, case):
    """mbt_ws_reference_beam draws the reference's particles (the three
    planes of generate_initial_sbunch_distribution2 on glibc's generator,
    as a fresh reference process seeds it) and the bunch offsets of
    generate_initial_general_distribution2; with the slicing they give the
    reference manager's starting slices bit for bit."""
    g = _golden(case)
    w, bucket, _ = _product(tmp_path, case)
    soa, off = api.SliceModel.reference_beam(w, len(bucket))
    assert np.array_equal(soa, g["particles"])
    _, _, cm4 = api.SliceModel.slice_beam(w, soa)
    assert np.array_equal(api.SliceModel.initial_slices(w, cm4, off), g["slices0"])


def test_bunch_model_probe(tmp_path, libmbt):
    """mbt_config_bunch_model tells the drop-in executable which model a
    file asks for."""
    L = api.lib()
    assert L.mbt_config_bunch_model(slice_conf(tmp_path, "train").encode()) == 1
    assert L.mbt_config_bunch_model(os.path.join(os.path.dirname(os.path.abspath(__file__)), "confs",
                                                 "uniform_fill.conf").encode()) == 0
    assert L.mbt_config_bunch_model(str(tmp_path / "missing.conf").encode()) < 0


def test_oracle_matches_golden_uneven_fill(tmp_path, libmbt):
    """The 321-bunch uneven fill (gaps, a 5 nC camshaft bunch, lognormal
    charges): two turns of the oracle equal the reference's bit for bit."""
    g = _golden("uneven")
    w, bucket, ib = _product(tmp_path, "train", **SLICE_UNEVEN)
    assert np.array_equal(bucket, g["bucket"]) and _same(ib, g["ibunch"])
    o = binding.OracleSlices(w, bucket, ib, g["npop"], g["nofe"])
    o.set_slices(g["slices0"])
    out = o.run(SLICE_UNEVEN_TURNS)
    for name, got in zip(("cm", "ion", "zcm", "stats"), out):
        assert _same(got, g[name]), name
    assert _same(o.slices_state(), g["slices"])


def test_writer_own_ampinv(tmp_path, libmbt):
    """With MBT_WRITER_OWN_AMPINV every per-monitor ampinv file lists each
    bunch's own invariants (the reference's history indexing otherwise
    shows other bunches' entries after the first monitor)."""
    g = _golden("train")
    w, bucket, ib = _product(tmp_path, "train", NrevTot=30, NrevMon=10)
    o = binding.OracleSlices(w, bucket, ib, g["npop"], g["nofe"])
    o.set_slices(g["slices0"])
    cm, ion, zcm, st = o.run(30)
    out = tmp_path / "own"
    out.mkdir()
    wr = api.SliceWriter(str(out), w, bucket, own_ampinv=True)
    wr.turns(ion, zcm, st)
    wr.close()
    for m, turn in enumerate((1, 11, 21)):
        rows = [l.split() for l in (out / ("ampinv_VER_%d.dat" % turn)).read_text().splitlines()[2:]]
        assert [int(r[0]) for r in rows] == list(bucket)
        got = np.array([[float(r[1]), float(r[2])] for r in rows])
        want = np.stack([st[m, :, 17], st[m, :, 14]], axis=1)
        assert np.allclose(got, want, rtol=1e-7, atol=0)


def test_slicing_edge_particles(tmp_path, libmbt):
    """Particles far outside the window, on slice edges, with NaN time or
    huge transverse offsets: the product's slicing equals the restatement's
    (NaN and far-ahead particles go to slice 0, far-behind ones to the
    overflow cell, huge offsets to the grid's edge points)."""
    w, _, _ = _product(tmp_path, "train")
    rng = np.random.default_rng(4)
    n = 3000
    p = np.stack([rng.normal(0, w.sgmatau, n), rng.normal(0, 2e-4, n), rng.normal(0, 2e-5, n),
                  rng.normal(0, 1e-3, n), rng.normal(0, 1e-5, n), rng.normal(0, 1e-6, n)])
    edges = (7.0 - np.arange(0, 48) * 0.3) * w.sgmatau
    p[0, :48] = edges
    p[0, 48:52] = [np.nan, 1e3 * w.sgmatau, -1e3 * w.sgmatau, 7.0 * w.sgmatau]
    p[1, 60:70] = 1e3
    p[2, 70:80] = -1e3
    a = api.SliceModel.slice_beam(w, p)
    b = binding.slice_beam(w, p)
    for x, y in zip(a, b):
        assert _same(x, y)
    # the NaN and the far-ahead particle sit in slice 0, the far-behind one
    # in the overflow cell that npop does not count
    assert a[0][0] >= 2 and a[0].sum() < n


@pytest.mark.reference
def test_oracle_matches_reference_long_run(tmp_path, libmbt):
    """200 turns of the 10-bunch train with the wall and the ions on, the
    oracle beside the reference's own functions: bit for bit throughout."""
    if not binding.reference_available() and not os.path.exists(binding.REF_SO):
        pytest.skip("reference harness unavailable")
    path = slice_conf(tmp_path, "train", NrevTot=300, NrevMon=50)
    r = binding.ReferenceSlices(path)
    w, bucket, ib = _product(tmp_path, "train", NrevTot=300, NrevMon=50)
    o = binding.OracleSlices(w, bucket, ib, r.npop, r.nofe)
    o.set_slices(r.slices_state())
    a = r.run(200, w.base.nrev_mon)
    b = o.run(200)
    for name, x, y in zip(("cm", "ion", "zcm", "stats"), a, b):
        assert _same(x, y), name
    assert _same(r.slices_state(), o.slices_state())
