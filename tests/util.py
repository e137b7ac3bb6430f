"""Shared helpers of the test-suite: configuration fixtures and comparisons."""
import os

import numpy as np

from oracle.binding import conf_with

HERE = os.path.dirname(os.path.abspath(__file__))
CONFS = os.path.join(HERE, "confs")
GOLDEN = os.path.join(HERE, "golden")


def conf(name):
    return os.path.join(CONFS, name)


def small_conf(tmp_path, name, **overrides):
    """A copy of tests/confs/<name> with `key = value` overrides; the fill
    files of the uneven and beam-ion configurations are made absolute."""
    src = conf(name)
    text = open(src).read()
    for fill in ("uneven_fill.txt", "beam_ion_fill.txt"):
        if fill in text and "filling" not in overrides:
            overrides["filling"] = os.path.join(CONFS, fill)
    dst = os.path.join(str(tmp_path), name)
    return conf_with(src, dst, **overrides)


def add_keys(path, section, **keys):
    """Insert `key = value` lines at the top of a section (for optional keys
    the fixture files do not carry)."""
    text = open(path).read()
    lines = "".join("\n  %s = %s" % (k, v) for k, v in keys.items())
    text = text.replace("[%s]" % section, "[%s]" % section + lines, 1)
    with open(path, "w") as f:
        f.write(text)
    return path


def add_tracking_keys(path, **keys):
    return add_keys(path, "tracking", **keys)


def rw_short_conf(tmp_path, **over):
    """The single-bunch configuration with the short-range resistive wall
    in three planes on 64 bins of 0.16 sigma (sigma_tau = 50 ps): bins of
    about 100 s0 for an 11 mm copper chamber."""
    path = small_conf(tmp_path, "single_bunch.conf", EnableRW_short=1, Ncell=64, sgm_xtau=0.05, **over)
    return add_keys(path, "ring", rhorw=1.678e-8, beffL1=0.011, beffL2=0.011, beffH3=0.012, beffH4=0.012,
                    beffV3=0.009, beffV4=0.009)


def add_section(path, name, **keys):
    """Append a `[name]` section with `key = value` lines."""
    with open(path, "a") as f:
        f.write("\n[%s]\n" % name + "".join("  %s = %s\n" % (k, v) for k, v in keys.items()))
    return path


_TRAIN = {"Np": 100, "Nmlt": 2, "filling": "SINGLE10", "EnableQuantum": 0, "xxCM_offset": 0.05,
          "gendst_datafile_LON": "dist_LON.dat", "gendst_datafile_HOR": "dist_HOR.dat",
          "gendst_datafile_VER": "dist_VER.dat"}

# Output-file cases: (conf, overrides, [tracking] additions[, added
# sections]).  The distribution files are named relative to the working
# directory.  The scan cases put the statistics lines of NrevMon and of the
# scan boundaries out of step, as the reference's scan value history then
# is.
WRITER_CASES = {
    "single": ("single_bunch.conf",
               {"Np": 200, "NrevTot": 40, "NrevMon": 20, "xxCM_offset": 0.05, "zzCM_offset": 0.02,
                "gendst_datafile_LON": "dist_LON.dat", "gendst_datafile_HOR": "dist_HOR.dat",
                "gendst_datafile_VER": "dist_VER.dat"},
               {"EnableAmpinv_out": 1}),
    "train_rw": ("uniform_fill.conf",
                 {"Np": 100, "Nmlt": 2, "filling": "SINGLE10", "NrevTot": 30, "NrevMon": 10,
                  "EnableQuantum": 0, "xxCM_offset": 0.05,
                  "gendst_datafile_LON": "dist_LON.dat", "gendst_datafile_HOR": "dist_HOR.dat",
                  "gendst_datafile_VER": "dist_VER.dat"},
                 {"EnableAmpinv_out": 1, "NrevPotentialsOut": 15}),
    "scan_current": ("uniform_fill.conf", dict(_TRAIN, NrevTot=1, NrevMon=6),
                     {"EnableAmpinv_out": 1, "NrevPotentialsOut": 3},
                     {"scan": {"scan_type": 1, "Nscan": 3, "NrevScan": 8, "scan_start": 150.0,
                               "scan_step": 30.0}}),
    "scan_q": ("uniform_fill.conf", dict(_TRAIN, NrevTot=1, NrevMon=4),
               {"EnableAmpinv_out": 1, "NrevPotentialsOut": 2},
               {"scan": {"scan_type": 3, "Nscan": 2, "NrevScan": 6}}),
}


def writer_conf(tmp_path, case):
    name, over, add = WRITER_CASES[case][:3]
    path = small_conf(tmp_path, name, **dict(over))
    add_tracking_keys(path, **add)
    for sec, keys in (WRITER_CASES[case][3] if len(WRITER_CASES[case]) > 3 else {}).items():
        add_section(path, sec, **keys)
    return path


def coord_err(a, b):
    """Largest difference per coordinate, relative to that coordinate's rms
    spread in b (coordinates near zero have no meaningful relative error)."""
    a = np.asarray(a).reshape(6, -1)
    b = np.asarray(b).reshape(6, -1)
    out = np.zeros(6)
    for k in range(6):
        scale = np.std(b[k])
        if scale == 0:
            scale = max(np.max(np.abs(b[k])), 1e-300)
        out[k] = np.max(np.abs(a[k] - b[k])) / scale if a[k].size else 0.0
    return out


def stats_err(a, b):
    """Statistics histories: centroids relative to the rms of the same
    plane, rms values relative to themselves (12 columns, see mbt.h)."""
    a = np.asarray(a)
    b = np.asarray(b)
    err = np.zeros(a.shape[:-1] + (12,))
    for k in range(3):
        for mean_col, rms_col in ((k, 3 + k), (6 + k, 9 + k)):
            scale = np.maximum(np.abs(b[..., rms_col]), 1e-300)
            err[..., mean_col] = np.abs(a[..., mean_col] - b[..., mean_col]) / scale
            err[..., rms_col] = np.abs(a[..., rms_col] - b[..., rms_col]) / scale
    return err


def centroid_err(a, b):
    """Centroid histories relative to their own size: for every bunch and
    plane (position and slope means, columns 0-2 and 6-8), the largest
    difference over the turns divided by max(largest |centroid| of b over
    the turns, 1e-6 x that plane's rms).  Statistics arrays are
    [turns, bunches, 12] (or [bunches, 12] for one turn)."""
    a = np.asarray(a, dtype=float)
    b = np.asarray(b, dtype=float)
    if a.ndim == 2:
        a, b = a[None], b[None]
    out = np.zeros(b.shape[1:-1] + (6,))
    for j, (mean_col, rms_col) in enumerate(((0, 3), (1, 4), (2, 5), (6, 9), (7, 10), (8, 11))):
        amp = np.max(np.abs(b[..., mean_col]), axis=0)
        floor = 1e-6 * np.max(np.abs(b[..., rms_col]), axis=0)
        scale = np.maximum(np.maximum(amp, floor), 1e-300)
        out[..., j] = np.max(np.abs(a[..., mean_col] - b[..., mean_col]), axis=0) / scale
    return out


# Slice model (BunchModel = STRONG) cases: ten consecutive bunches of
# 0.5 nC with the long-range resistive wall; and six bunches followed by a
# 5 nC bunch 195 buckets later (ions drift across the gap), 41 slices, the
# resistive-wall trigger on.
SLICE_CASES = {
    "train": {"Np": 2000, "NrevTot": 40},
    "gaps": {"Np": 2000, "NrevTot": 40, "Nslc": 20, "filling": os.path.join(CONFS, "short_fill.txt"),
             "Iring": 3.38},
}
SLICE_TURNS = 30
# the 321-bunch uneven fill (three trains, camshaft bunch, lognormal charges)
# with 21 slices, two turns
SLICE_UNEVEN = {"Np": 2000, "NrevTot": 10, "Nslc": 10, "filling": os.path.join(CONFS, "uneven_fill.txt"),
                "Iring": 150.0}
SLICE_UNEVEN_TURNS = 2
# the drop-in executable's slice-model run: 60 turns, monitors every 20
SLICE_CLI_OVER = {"Np": 2000, "NrevTot": 60, "NrevMon": 20}


def slice_conf(tmp_path, case, **over):
    """A copy of tests/confs/slice_fbii.conf for SLICE_CASES[case]."""
    keys = dict(SLICE_CASES[case])
    keys.update(over)
    trigger = keys.pop("triggerRW", 1 if case == "gaps" else None)
    path = conf_with(conf("slice_fbii.conf"), os.path.join(str(tmp_path), "slice_%s.conf" % case), **keys)
    if trigger is not None:
        add_tracking_keys(path, triggerRW=trigger)
    return path
