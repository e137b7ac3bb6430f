"""Slice model (BunchModel = STRONG) with fast beam-ion interaction on the
GPU (mbt_ws.h) against the oracle (oracle/ws_oracle.c, itself bit-exact
with the reference's functions, tests/test_slice_model.py).

The device reproduces the oracle's arithmetic operation by operation
(libmbt's mbt_ws.cu is built without multiply-add contraction); what
differs is the last bits of sin, exp and w(z) on the device and the
summation order of the ion kick and ion centroid sums (a fixed tree on the
device, sequential in the reference).  Tolerances: 1e-9 of each output's
largest magnitude after 30 turns; 1e-12 for the field grids and ions of
one turn."""
import os

import numpy as np
import pytest

from mbtrack_b200 import api
from oracle import binding
from tests.util import GOLDEN, SLICE_CASES, SLICE_TURNS, SLICE_UNEVEN, SLICE_UNEVEN_TURNS, slice_conf

pytestmark = pytest.mark.gpu


def _setup(tmp_path, case, **over):
    w, bucket, frac = api.SliceModel.config(slice_conf(tmp_path, case, **over))
    L = api.lib()
    ib = np.array([L.mbt_bunch_current(w.base, len(bucket), float(f)) * 1e3 for f in frac])
    g = np.load(os.path.join(GOLDEN, "slice_fbii_%s.npz" % case))
    npop, nofe, _ = api.SliceModel.slice_beam(w, g["particles"])
    return w, bucket, ib, npop, nofe, g


def _close(got, want, rel, name):
    assert np.array_equal(np.isnan(got), np.isnan(want)), name
    if want.size == 0 or np.isnan(want).all():
        return 0.0
    scale = np.nanmax(np.abs(want))
    err = np.nanmax(np.abs(got - want)) if want.size else 0.0
    assert err <= rel * scale, "%s: %.3e of %.3e" % (name, err, scale)
    return err / scale if scale else 0.0


@pytest.mark.parametrize("case", sorted(SLICE_CASES))
def test_device_matches_oracle(tmp_path, cuda_device, case):
    w, bucket, ib, npop, nofe, g = _setup(tmp_path, case)
    dev = api.SliceModel(w, bucket, ib, npop, nofe)
    dev.load_slices(g["slices0"])
    o = binding.OracleSlices(w, bucket, ib, npop, nofe)
    o.set_slices(g["slices0"])
    # one turn: field grids and the bunches' own ions
    a = dev.run(1)
    b = o.run(1)
    for ibn in range(len(bucket)):
        e1, i1 = dev.bunch_fields(ibn)
        e2, i2 = o.bunch_fields(ibn)
        _close(e1, e2, 1e-12, "fields %d" % ibn)
        _close(i1, i2, 1e-12, "ions %d" % ibn)
    for name, x, y in zip(("cm", "ion", "zcm", "stats"), a, b):
        _close(x, y, 1e-12, name)
    # the rest of the 30 turns, against the oracle and the reference's fixture
    a2 = dev.run(SLICE_TURNS - 1)
    b2 = o.run(SLICE_TURNS - 1)
    worst = {}
    for k, name in enumerate(("cm", "ion", "zcm", "stats")):
        x = np.concatenate([a[k], a2[k]])
        y = np.concatenate([b[k], b2[k]])
        worst[name] = _close(x, y, 1e-9, name)
        _close(x, g[name], 1e-9, name + " (reference)")
    _close(dev.slices(), o.slices_state(), 1e-9, "slices")
    print(case, "relative deviations:", worst)


def test_device_runs_repeat_bit_for_bit(tmp_path, cuda_device):
    """Fixed reduction order: two contexts give identical outputs."""
    w, bucket, ib, npop, nofe, g = _setup(tmp_path, "train")
    outs = []
    for _ in range(2):
        dev = api.SliceModel(w, bucket, ib, npop, nofe)
        dev.load_slices(g["slices0"])
        outs.append(dev.run(12) + (dev.slices(),))
        dev.close()
    for x, y in zip(*outs):
        assert np.array_equal(x, y, equal_nan=True)


@pytest.mark.parametrize("over", [{"EnableFBII": 0}, {"EnableRW_long": 0}, {"NrevMon": 1}, {"Nslc": 3}],
                         ids=["no_fbii", "no_rw", "mon_every_turn", "nslc3_all_in_overflow"])
def test_device_variants(tmp_path, cuda_device, over):
    """Beam-ion off (no ions: NaN ion centroid, resistive wall only),
    resistive wall off, statistics every turn, and the reference's default
    Nslc = 3, where every particle falls in the overflow cell (empty slices:
    NaN centroids, as in the reference)."""
    w, bucket, ib, npop, nofe, g = _setup(tmp_path, "train", **over)
    soa, off = api.SliceModel.reference_beam(w, len(bucket))
    s0 = api.SliceModel.initial_slices(w, api.SliceModel.slice_beam(w, soa)[2], off)
    dev = api.SliceModel(w, bucket, ib, npop, nofe)
    dev.load_slices(s0)
    o = binding.OracleSlices(w, bucket, ib, npop, nofe)
    o.set_slices(s0)
    a = dev.run(15)
    b = o.run(15)
    for name, x, y in zip(("cm", "ion", "zcm", "stats"), a, b):
        _close(x, y, 1e-9, name)
    if not w.fbii:
        assert np.isnan(a[1]).all()


def test_chunked_outputs(tmp_path, cuda_device):
    """A run longer than one block of host outputs (256 turns) equals the
    same turns run in pieces."""
    w, bucket, ib, npop, nofe, g = _setup(tmp_path, "gaps", NrevTot=600)
    d1 = api.SliceModel(w, bucket, ib, npop, nofe)
    d1.load_slices(g["slices0"])
    a = d1.run(300)
    d2 = api.SliceModel(w, bucket, ib, npop, nofe)
    d2.load_slices(g["slices0"])
    parts = [d2.run(n) for n in (100, 7, 193)]
    for k in range(4):
        assert np.array_equal(a[k], np.concatenate([p[k] for p in parts]), equal_nan=True)
    assert d2.turn == 300


def _np_interp(Ex, Ey, icell, G, ax, az, xs, ys):
    """get_linearly_interpolated_Efields (fbi_weakstrong.c:454-580) in
    Python floats: IEEE division, the reference's operand order."""
    off = (G - 1) // 2
    out = np.zeros((len(xs), 2))
    for i, (xx, yy) in enumerate(zip(xs, ys)):
        k1x, k1z = int(xx / ax), int(yy / az)
        if yy >= 0:
            k2z = k1z + 1 if k1z < off else k1z
            k1z, k2z = min(k1z, off), min(k2z, off)
        else:
            k2z = k1z - 1 if k1z > -off else k1z
            k1z, k2z = max(k1z, -off), max(k2z, -off)
        if xx >= 0:
            k2x = k1x + 1 if k1x < off else k1x
            k1x, k2x = min(k1x, off), min(k2x, off)
        else:
            k2x = k1x - 1 if k1x > -off else k1x
            k1x, k2x = max(k1x, -off), max(k2x, -off)
        b = icell * G
        i1 = (b + k1x + off) * G + k1z + off
        i2 = (b + k2x + off) * G + k1z + off
        i3 = (b + k1x + off) * G + k2z + off
        i4 = (b + k2x + off) * G + k2z + off
        fx = (xx - k1x * ax) / ax
        fz = (yy - k1z * az) / az
        r = []
        for E in (Ex, Ey):
            if xx >= 0:
                e5 = E[i1] + fx * (E[i2] - E[i1])
                e6 = E[i3] + fx * (E[i4] - E[i3])
            else:
                e5 = E[i1] - fx * (E[i2] - E[i1])
                e6 = E[i3] - fx * (E[i4] - E[i3])
            r.append(e5 + fz * (e6 - e5) if yy >= 0 else e5 - fz * (e6 - e5))
        out[i] = r
    return out


def test_device_interpolation_bit_exact(tmp_path, cuda_device):
    """The device's interpolation, with its division by the grid step done
    as a multiplication by the reciprocal plus two residual corrections,
    equals the reference's expression with IEEE division bit for bit: at
    random points, on and one ulp either side of every grid line, far
    outside the grid and at zero of both signs."""
    w, bucket, ib, npop, nofe, g = _setup(tmp_path, "train")
    dev = api.SliceModel(w, bucket, ib, npop, nofe)
    dev.load_slices(g["slices0"])
    dev.run(2, outputs=False)
    ax, az = w.agABSx, w.agABSz
    rng = np.random.default_rng(11)
    lines = np.arange(-4, 5)
    xs = [rng.uniform(-4, 4, 1500) * ax, rng.uniform(-300, 300, 200) * ax,
          np.nextafter(lines * ax, np.inf), np.nextafter(lines * ax, -np.inf), lines * ax,
          np.array([0.0, -0.0, 0.0, -0.0])]
    ys = [rng.uniform(-4, 4, 1500) * az, rng.uniform(-300, 300, 200) * az,
          np.nextafter(lines * az, -np.inf), np.nextafter(lines * az, np.inf), lines * az,
          np.array([0.0, -0.0, -0.0, 0.0])]
    x = np.concatenate(xs)
    y = np.concatenate(ys)
    for ibn, icell in ((0, 23), (3, 10), (9, 30)):
        exey, _ = dev.bunch_fields(ibn)
        got = dev.interp(ibn, icell, x, y)
        want = _np_interp(exey[:, 0], exey[:, 1], icell, w.ngrid, ax, az, x, y)
        assert np.array_equal(got, want), np.abs(got - want).max()


def test_cli_slice_model_writes_reference_files(tmp_path, cuda_device):
    """mbtrack-gpu on a BunchModel = STRONG file: the reference's generated
    bunch and slicing, the device turn, and the files of the reference's
    slice-model manager (its own writers, tests/golden/slice_fbii_cli.npz):
    motion files every turn, ampinv files every NrevMon, the means and the
    generated distribution.  Numbers may sit one unit apart in the last
    printed digit (tests/test_gpu_cli.py's rule); nothing else may differ."""
    import subprocess
    from mbtrack_b200 import build
    from tests.test_gpu_cli import compare_text
    from tests.util import SLICE_CLI_OVER
    build.build()
    over = dict(SLICE_CLI_OVER)
    for pl in ("LON", "HOR", "VER"):
        over["gendst_datafile_" + pl] = str(tmp_path / ("gendst_" + pl))
    conf = slice_conf(tmp_path, "train", **over)
    work = tmp_path / "work"
    work.mkdir()
    r = subprocess.run([build.CLI, conf, str(work)], cwd=str(work), capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr + r.stdout
    assert "Starting multi bunch tracking..." in r.stdout and " done" in r.stdout
    z = np.load(os.path.join(GOLDEN, "slice_fbii_cli.npz"))
    ref = {k: str(z[k]) for k in z.files}
    ours = sorted(os.listdir(work))
    assert ours == sorted(k for k in ref if not k.startswith("gendst_"))
    flips, total, bad = 0, 0, []
    for f in ours + ["gendst_LON", "gendst_HOR", "gendst_VER"]:
        p = work / f if not f.startswith("gendst_") else tmp_path / f
        n, b = compare_text(f, p.read_text(), ref[f])
        bad += b
        flips += n
        total += len(ref[f].split())
    assert not bad, "\n".join(bad[:30])
    assert flips <= max(3, total // 10000), "%d numbers one digit apart of %d tokens" % (flips, total)


def test_device_matches_reference_uneven_fill(tmp_path, cuda_device):
    """The 321-bunch uneven fill: two device turns against the reference's
    own (tests/golden/slice_fbii_uneven.npz)."""
    g = np.load(os.path.join(GOLDEN, "slice_fbii_uneven.npz"))
    w, bucket, frac = api.SliceModel.config(slice_conf(tmp_path, "train", **SLICE_UNEVEN))
    L = api.lib()
    ib = np.array([L.mbt_bunch_current(w.base, len(bucket), float(f)) * 1e3 for f in frac])
    dev = api.SliceModel(w, bucket, ib, g["npop"], g["nofe"])
    dev.load_slices(g["slices0"])
    out = dev.run(SLICE_UNEVEN_TURNS)
    for name, x in zip(("cm", "ion", "zcm", "stats"), out):
        _close(x, g[name], 1e-11, name)
    _close(dev.slices(), g["slices"], 1e-11, "slices")


def test_checkpoint_resume(tmp_path, cuda_device):
    """A slice-model run saved after 12 turns and resumed in a fresh
    context continues bit for bit; a truncated file is refused."""
    w, bucket, ib, npop, nofe, g = _setup(tmp_path, "train")
    ck = str(tmp_path / "ws.ckpt")
    a = api.SliceModel(w, bucket, ib, npop, nofe)
    a.load_slices(g["slices0"])
    a.run(12)
    a.checkpoint_save(ck)
    ra = a.run(8)
    b = api.SliceModel(w, bucket, ib, npop, nofe)
    b.checkpoint_load(ck)
    assert b.turn == 12
    rb = b.run(8)
    for x, y in zip(ra, rb):
        assert np.array_equal(x, y, equal_nan=True)
    data = open(ck, "rb").read()
    bad = str(tmp_path / "bad.ckpt")
    open(bad, "wb").write(data[:-9])
    with pytest.raises(api.MbtError):
        b.checkpoint_load(bad)
    assert b.turn == 20


def test_growth_rate_against_the_per_particle_stage(cuda_device):
    """The slice model (BunchModel = STRONG, the reference's fast beam-ion
    interaction) and the per-particle weak-strong beam-ion stage are two
    models of the same instability; on one shared configuration (the
    200-bunch train, CO at the slice model's pressure over the whole ring,
    no wall, no chromaticity, no radiation noise) their vertical growth
    rates agree within a factor of 3 with the physical (thin-lens) ion kick
    of the slice model, which grows the slower of the two (its ions sit on
    a coarse grid around the slice centroids and kick rigid slices); the
    reference's ion kick factor 1e2 makes the slice model grow far faster."""
    import bench
    r = bench.slice_growth_compare(3000)
    thin, ref, per = r["slice_kick_factor_1"], r["slice_kick_factor_100"], r["per_particle"]
    for x in (thin, per):
        assert x["window"] is not None and x["rate_per_turn"] > 0, x
    assert 1.0 <= per["rate_per_turn"] / thin["rate_per_turn"] <= 3.0, (per["rate_per_turn"], thin["rate_per_turn"])
    # after 100 turns the reference's kick factor has grown the motion far beyond the thin-lens run
    assert ref["amplitude_every_100_turns"][1] > 10 * thin["amplitude_every_100_turns"][1], (ref, thin)
