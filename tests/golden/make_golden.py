"""Generates the golden fixtures of tests/golden/ by running the reference's
own sources (compiled unmodified into oracle/_ref/libmbtref.so by
oracle/Makefile from the reference tree) through oracle/ref_harness.c.

    python tests/golden/make_golden.py

Each case stores the reference's derived parameters, Green's functions,
initial beam and statistics, per-turn statistics, final beam and (with
noise) the deviates it drew.  A w(z) grid evaluated by the reference's
complex_errorfunc_wofz_algo680 (physic.c:75-301) is stored too.  The
fixtures let the oracle be checked on machines without the reference tree.
"""
import ctypes
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from mbtrack_b200.abi import params_to_dict  # noqa: E402
from oracle.binding import Reference, build_reference, conf_with  # noqa: E402

CONFS = os.path.join(ROOT, "tests", "confs")

# name -> (conf file, overrides, turns, record deviates)
CASES = {
    "single_noiseoff": ("single_bunch.conf", {"Np": 2000, "xxCM_offset": 0.05, "zzCM_offset": 0.02,
                                             "xtauCM_offset": 0.002}, 40, False),
    "single_noise": ("single_bunch.conf", {"Np": 1000, "xxCM_offset": 0.05, "EnableQuantum": 1}, 10, True),
    "train_rw_hom": ("uniform_fill.conf", {"Np": 200, "Nmlt": 3, "filling": "SINGLE10",
                                           "EnableQuantum": 0, "xxCM_offset": 0.05}, 12, False),
    "feedback_hc": ("feedback_hc.conf", {"filling": os.path.join(CONFS, "short_fill.txt")}, 15, False),
}


def run_case(name, conf, over, turns, record, tmp):
    path = conf_with(os.path.join(CONFS, conf), os.path.join(tmp, name + ".conf"), **over)
    R = Reference(path)
    init = [R.get_particles(i) for i in range(R.nb)]
    st0 = R.prepare()
    Gl, Gv, Gh, planes = R.greens()
    p = R.params()
    per = 1 + 2 * (p.track_plane[2] != 0) + 2 * (p.track_plane[1] != 0)
    cap = int(turns * per * R.np.sum()) if (record and p.quantum) else 0
    if cap:
        st, dev = R.run(turns, record=True, dev_cap=cap)
    else:
        st, dev = R.run(turns), np.zeros(0, dtype=np.float32)
    final = [R.get_particles(i) for i in range(R.nb)]
    vrf_phi, phasor = R.state(0)
    out = os.path.join(HERE, name + ".npz")
    np.savez_compressed(
        out, bucket=R.bucket, np=R.np, ib=R.ib, Gl=Gl, Gv=Gv, Gh=Gh,
        init=np.concatenate([a.ravel() for a in init]), init_stats=st0, stats=st,
        final=np.concatenate([a.ravel() for a in final]), deviates=dev, vrf_phi=vrf_phi,
        phasor=phasor, params=json.dumps(params_to_dict(p)),
        conf=conf, overrides=json.dumps({k: str(v) for k, v in over.items()}),
        deviates_exact=R.deviates_exact())
    print(name, "->", out, os.path.getsize(out), "bytes")


def wofz_grid():
    lib = ctypes.CDLL(build_reference())
    f = lib.complex_errorfunc_wofz_algo680
    f.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.POINTER(ctypes.c_double)]
    f.restype = ctypes.c_int
    rng = np.random.default_rng(680)
    pts = [rng.uniform(-8, 8, (1500, 2)), rng.uniform(-0.6, 0.6, (500, 2)),
           rng.uniform(-30, 30, (300, 2)), np.array([[0, 0], [1e-3, 0], [3.0, 0], [0, 2.0], [0, -2.0],
                                                     [5.9, 0.001], [-5.9, -0.001], [0.3, 1e-12]])]
    xy = np.concatenate(pts)
    re = np.zeros(len(xy))
    im = np.zeros(len(xy))
    fl = np.zeros(len(xy), dtype=np.int32)
    w = (ctypes.c_double * 2)()
    for i, (x, y) in enumerate(xy):
        fl[i] = f(float(x), float(y), w)
        re[i], im[i] = w[0], w[1]
    out = os.path.join(HERE, "wofz_grid.npz")
    np.savez_compressed(out, x=xy[:, 0], y=xy[:, 1], re=re, im=im, flag=fl)
    print("wofz grid ->", out, os.path.getsize(out), "bytes")


def main():
    import tempfile
    tmp = tempfile.mkdtemp()
    for name, (conf, over, turns, record) in CASES.items():
        run_case(name, conf, over, turns, record, tmp)
    wofz_grid()


if __name__ == "__main__":
    main()
