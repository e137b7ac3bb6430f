"""The output files (mbt_writer_*, mbt_config_output, mbt_reference_beam):
libmbt's writer, given the statistics stream of a reference run, writes the
reference's files byte for byte.

The expected files come from the reference's own printing functions
(bunch_stats_fprintf bunch.c:792-804, worker_weak_stat_output bunch.c:773-789,
bunch_weak_writeout_ampinv bunch.c:588-640, weak_bunch_writeout_tbtbbb
bunch_weak.c:343-387, weak_bunch_writeout_mean_ampinv bunch_weak.c:390-447,
weak_writeout_bunch_distribution bunch_weak.c:296-332, the potentials of
transform_weak.c:735-768), run through oracle/ref_harness.c: live when the
reference tree is present, from tests/golden/writer_*.npz otherwise.
"""
import json
import os

import numpy as np
import pytest

from mbtrack_b200 import api
from tests.golden_cases import CASES, Case
from tests.util import CONFS, GOLDEN, WRITER_CASES, small_conf, writer_conf


def golden(case):
    z = np.load(os.path.join(GOLDEN, "writer_%s.npz" % case), allow_pickle=False)
    d = {k: z[k] for k in z.files}
    d["files"] = json.loads(str(z["files"]))
    return d


def parse_potentials(text, nc):
    """(rev, 7 x nc potential terms) per event of a potentials file."""
    rows = [l.split() for l in text.splitlines() if l.strip() and not l.startswith(" #")]
    out = []
    for e in range(len(rows) // nc):
        blk = rows[e * nc:(e + 1) * nc]
        pot = np.zeros((7, nc))
        for j, r in enumerate(blk):
            pot[0, j], pot[1, j], pot[2, j] = float(r[3]), float(r[4]), float(r[8])
            if len(r) > 9:
                pot[3, j], pot[4, j] = float(r[9]), float(r[10])
            if len(r) > 11:
                pot[5, j], pot[6, j] = float(r[11]), float(r[12])
        out.append((int(blk[0][0]) - 1, pot))
    return out


def write_from_stream(tmp_path, case, g, own_ampinv=False):
    """Feed a reference run's statistics stream to libmbt's writer."""
    conf = writer_conf(tmp_path, case)
    C = api.Config(conf)
    o, bout = C.output()
    work = os.path.join(str(tmp_path), "mbt")
    os.makedirs(work)
    for pl, tag in enumerate(("LON", "HOR", "VER")):
        o.gendst_file[pl].value = os.path.join(work, "dist_%s.dat" % tag).encode()
    W = api.Writer(work, C.params, o, bout, C.bucket, g["ib"], own_ampinv=own_ampinv)
    W.wakes(C.Gl, C.Gv, C.Gh)
    W.begin(g["init_stats"])
    outb = [i for i in range(len(C.bucket)) if C.bucket[i] in set(bout.tolist())]
    pots = {i: dict(parse_potentials(g["files"].get("potentials_bunch_%d.dat" % C.bucket[i], ""),
                                     C.params.ncell)) for i in outb}
    for rev in range(C.params.nrev_tot):
        if W.potentials_due(rev):
            for i in outb:
                W.potentials(i, rev, pots[i][rev], g["vrfphi"][rev, i, 0], g["vrfphi"][rev, i, 1])
        W.turns(g["stats"][rev:rev + 1], g["ampinv"][rev:rev + 1])
    W.end(g["end_stats"])
    if outb:
        W.distribution(outb[0], g["final"])
    W.close()
    return work, C


@pytest.mark.parametrize("case", sorted(WRITER_CASES))
def test_writer_reproduces_reference_files(tmp_path, case):
    g = golden(case)
    work, _ = write_from_stream(tmp_path, case, g)
    ours = sorted(os.listdir(work))
    assert ours == sorted(g["files"]), (ours, sorted(g["files"]))
    for f in ours:
        text = open(os.path.join(work, f)).read()
        assert text == g["files"][f], "%s differs from the reference's" % f


def test_writer_own_ampinv_indexing(tmp_path):
    """MBT_WRITER_OWN_AMPINV prints each bunch's own invariants; the default
    reproduces the reference's monitor + bucket indexing (bunch.c:599-601)."""
    g = golden("train_rw")
    work, C = write_from_stream(tmp_path, "train_rw", g, own_ampinv=True)
    nb = len(C.bucket)
    mon = C.params.nrev_mon
    for rev in range(mon - 1, C.params.nrev_tot, mon):
        rows = [l.split() for l in open(os.path.join(work, "ampinv_HOR_%d.dat" % (rev + 1)))
                if not l.startswith("#")]
        assert len(rows) == nb
        for b, r in enumerate(rows):
            assert int(r[0]) == C.bucket[b]
            assert float(r[1]) == pytest.approx(g["ampinv"][rev, b, 4], rel=1e-8, abs=1e-300)
            assert float(r[2]) == pytest.approx(g["ampinv"][rev, b, 1], rel=1e-8, abs=1e-300)
    # the first monitor agrees with the reference's indexing, later ones not
    assert open(os.path.join(work, "ampinv_HOR_%d.dat" % mon)).read() == g["files"]["ampinv_HOR_%d.dat" % mon]


def test_writer_rejects_misuse(tmp_path):
    g = golden("single")
    conf = writer_conf(tmp_path, "single")
    C = api.Config(conf)
    o, bout = C.output()
    work = str(tmp_path)
    W = api.Writer(work, C.params, o, bout, C.bucket, g["ib"])
    with pytest.raises(api.MbtError):
        W.turns(g["stats"][:1], g["ampinv"][:1])          # before begin
    W.begin(g["init_stats"])
    with pytest.raises(api.MbtError):
        W.end(g["end_stats"])                               # turns missing
    with pytest.raises(api.MbtError):
        W.turns(np.zeros((C.params.nrev_tot + 1, 1, 12)), np.zeros((C.params.nrev_tot + 1, 1, 6)))
    W.close()
    with pytest.raises(api.MbtError):
        api.Writer(os.path.join(work, "no", "such", "dir"), C.params, o, bout, C.bucket, g["ib"])


@pytest.mark.parametrize("name", CASES)
def test_reference_beam_matches_golden(tmp_path, name):
    """mbt_reference_beam reproduces the reference's generated distribution
    (weak_generate_bunch_distribution, c_fnorm with glibc rand()) bit for
    bit, for every bunch of every golden case."""
    c = Case(name)
    C = api.Config(c.conf_file(tmp_path))
    beams = C.reference_beam()
    init = c.bunch_slices(c.init)
    assert len(beams) == len(init)
    for b, (ours, ref) in enumerate(zip(beams, init)):
        assert np.array_equal(ours, ref), "bunch %d" % b


def test_config_output_lists(tmp_path):
    """Output buckets of e_beam_setup (input.c:1316-1426) and of a filling
    file's third column (e_beam_fileread input.c:1445-1512)."""
    expect = {"SINGLE": [0], "SINGLE3": [0, 1, 2], "SINGLE10": [0, 4, 9], "SINGLE20": [0, 9, 19],
              "UNIFORM": [0], "ONEFOURTH": [0, 52, 103], "ONETHIRD": [0, 69, 137],
              "TWOTHIRD": [0, 138, 276], "THREEFOURTH": [0, 156, 311], "EVENHALF": [0]}
    for fill, buckets in expect.items():
        conf = small_conf(tmp_path, "single_bunch.conf", filling=fill)
        C = api.Config(conf)
        o, bout = C.output()
        assert list(bout) == buckets, fill
        assert C.params.scan == 0 and C.params.nrev_scan == C.params.nrev_tot + 1
        assert o.ampinv_out == 0 and o.nrev_potentials_out == 0
        assert o.jobtitle == b"single"
    conf = small_conf(tmp_path, "uneven_fill.conf")
    o, bout = api.Config(conf).output()
    fill_file = [l.split() for l in open(os.path.join(CONFS, "uneven_fill.txt")) if l.strip()]
    marked = [int(r[0]) for r in fill_file if float(r[1]) > 0 and int(r[2]) != 0]
    assert len(marked) > 0 and list(bout) == marked


def test_writer_live_uneven_fill(tmp_path):
    """Live against the reference on an uneven fill with RF feedback: every
    file identical, except the ampinv lines for which the reference reads
    past its history array (entry monitor + bucket, bunch.c:599-601, or
    monitor x Nbunch + bucket, bunch_weak.c:415-428, beyond its
    NrevTot / NrevMon x Nbunch + 2 entries); the writer reads 0 there."""
    from oracle.binding import Reference, build_reference, reference_available
    if not reference_available() or build_reference() is None:
        pytest.skip("reference tree not present")
    from tests.util import add_tracking_keys, CONFS as confs
    tmp = str(tmp_path)
    ref_dir = os.path.join(tmp, "ref")
    os.makedirs(ref_dir)
    over = {"filling": os.path.join(confs, "short_fill.txt"), "Np": 200, "NrevTot": 30, "NrevMon": 10,
            "gendst_datafile_LON": os.path.join(ref_dir, "dist_LON.dat"),
            "gendst_datafile_HOR": os.path.join(ref_dir, "dist_HOR.dat"),
            "gendst_datafile_VER": os.path.join(ref_dir, "dist_VER.dat")}
    conf = add_tracking_keys(small_conf(tmp_path, "feedback_hc.conf", **over), EnableAmpinv_out=1)
    R = Reference(conf, workdir=ref_dir)
    st0 = R.prepare()
    st, ai, vp, end = R.run_files()
    first = [i for i in range(R.nb) if R.bucket[i] in set(R.output_info()["bunch_out"].tolist())]
    g = {"init_stats": st0, "stats": st, "ampinv": ai, "vrfphi": vp, "end_stats": end,
         "final": R.get_particles(first[0]).reshape(6, -1), "ib": R.ib,
         "files": {f: open(os.path.join(ref_dir, f)).read() for f in os.listdir(ref_dir)}}
    C = api.Config(conf)
    o, bout = C.output()
    work = os.path.join(tmp, "mbt")
    os.makedirs(work)
    for pl, tag in enumerate(("LON", "HOR", "VER")):
        o.gendst_file[pl].value = os.path.join(work, "dist_%s.dat" % tag).encode()
    W = api.Writer(work, C.params, o, bout, C.bucket, R.ib)
    W.wakes(C.Gl, C.Gv, C.Gh)
    W.begin(st0)
    outb = first
    pots = {i: dict(parse_potentials(g["files"]["potentials_bunch_%d.dat" % C.bucket[i]], C.params.ncell))
            for i in outb}
    for rev in range(C.params.nrev_tot):
        if W.potentials_due(rev):
            for i in outb:
                W.potentials(i, rev, pots[i][rev], vp[rev, i, 0], vp[rev, i, 1])
        W.turns(st[rev:rev + 1], ai[rev:rev + 1])
    W.end(end)
    W.distribution(outb[0], g["final"])
    W.close()
    assert sorted(os.listdir(work)) == sorted(g["files"])
    nb, rows = len(C.bucket), C.params.nrev_tot // C.params.nrev_mon
    bunch_of = {int(b): i for i, b in enumerate(C.bucket)}
    for f, ref_text in g["files"].items():
        ours = open(os.path.join(work, f)).read()
        if ours == ref_text:
            continue
        assert f.startswith("ampinv_"), f
        nhist = rows * nb + 2
        for lo, lr in zip(ours.splitlines(), ref_text.splitlines()):
            if lo == lr:
                continue
            if f.endswith("_mean.dat"):
                # bunch_weak.c:415-428: entry irevmon Nbunch + bucket
                irevmon = int(lo.split()[0]) // C.params.nrev_mon
                assert irevmon * nb + max(bunch_of) >= nhist, (f, lo, lr)
            else:
                irevmon = int(f.split("_")[2].split(".")[0]) // C.params.nrev_mon - 1
                jb = int(lo.split()[0])
                assert jb in bunch_of and irevmon + jb >= nhist, (f, lo, lr)
                assert float(lo.split()[1]) == 0.0 and float(lo.split()[2]) == 0.0
