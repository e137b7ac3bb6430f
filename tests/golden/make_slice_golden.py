"""Generates tests/golden/slice_fbii_<case>.npz: the reference's own slice
model with fast beam-ion interaction (manager_/worker_weakstrong.c,
rw_weakstrong.c, fbi_weakstrong.c; BunchModel = STRONG), run by
oracle/ref_ws_harness.c on the configurations of SLICE_CASES (tests/util.py).

Each file holds the particles the reference slices, its slicing (npop,
nofe), the fill (bucket, ibunch [mA]), the initial slice state and the
per-turn outputs of TURNS turns (cm, ion, zcm, stats) with the final slice
state (slice_fbii_uneven.npz: the 321-bunch fill of SLICE_UNEVEN, two turns,
without the particles).  slice_fbii_cli.npz holds the files the reference's manager writes
for SLICE_CLI_OVER (its writers called by the harness): name -> text.

    python tests/golden/make_slice_golden.py
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import binding  # noqa: E402
from tests.util import SLICE_CASES, SLICE_CLI_OVER, SLICE_TURNS, SLICE_UNEVEN, SLICE_UNEVEN_TURNS, slice_conf  # noqa: E402


def main():
    with tempfile.TemporaryDirectory() as tmp:
        path = slice_conf(tmp, "train", **SLICE_UNEVEN)
        r = binding.ReferenceSlices(path)
        s0 = r.slices_state()
        cm, ion, zcm, st = r.run(SLICE_UNEVEN_TURNS, r.params().base.nrev_mon)
        out = os.path.join(HERE, "slice_fbii_uneven.npz")
        np.savez_compressed(out, npop=r.npop, nofe=r.nofe, bucket=r.bucket, ibunch=r.ibunch, slices0=s0, cm=cm,
                            ion=ion, zcm=zcm, stats=st, slices=r.slices_state())
        print(out, r.nb, "bunches", r.slices, "slices")
    for case in SLICE_CASES:
        with tempfile.TemporaryDirectory() as tmp:
            path = slice_conf(tmp, case)
            r = binding.ReferenceSlices(path)
            s0 = r.slices_state()
            cm, ion, zcm, st = r.run(SLICE_TURNS, r.params().base.nrev_mon)
            out = os.path.join(HERE, "slice_fbii_%s.npz" % case)
            np.savez_compressed(out, particles=r.particles(), npop=r.npop, nofe=r.nofe, bucket=r.bucket,
                                ibunch=r.ibunch, slices0=s0, cm=cm, ion=ion, zcm=zcm, stats=st,
                                slices=r.slices_state())
            print(out, r.nb, "bunches", r.slices, "slices")
    with tempfile.TemporaryDirectory() as tmp:
        over = dict(SLICE_CLI_OVER)
        for pl in ("LON", "HOR", "VER"):
            over["gendst_datafile_" + pl] = os.path.join(tmp, "gendst_" + pl)
        path = slice_conf(tmp, "train", **over)
        work = os.path.join(tmp, "work")
        os.mkdir(work)
        r = binding.ReferenceSlices(path, workdir=work)
        r.files(True)
        r.write_distribution()
        r.run(over["NrevTot"], over["NrevMon"])
        r.finish()
        files = {n: open(os.path.join(work, n)).read() for n in sorted(os.listdir(work))}
        for pl in ("LON", "HOR", "VER"):
            files["gendst_" + pl] = open(os.path.join(tmp, "gendst_" + pl)).read()
        out = os.path.join(HERE, "slice_fbii_cli.npz")
        np.savez_compressed(out, **{k: np.array(v) for k, v in files.items()})
        print(out, len(files), "files")


if __name__ == "__main__":
    main()
