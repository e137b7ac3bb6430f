"""Generates tests/golden/slice_fbii_<case>.npz: the reference's own slice
model with fast beam-ion interaction (manager_/worker_weakstrong.c,
rw_weakstrong.c, fbi_weakstrong.c; BunchModel = STRONG), run by
oracle/ref_ws_harness.c on the configurations of SLICE_CASES (tests/util.py).

Each file holds the particles the reference slices, its slicing (npop,
nofe), the fill (bucket, ibunch [mA]), the initial slice state and the
per-turn outputs of TURNS turns (cm, ion, zcm, stats) with the final slice
state.

    python tests/golden/make_slice_golden.py
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import binding  # noqa: E402
from tests.util import SLICE_CASES, SLICE_TURNS, slice_conf  # noqa: E402


def main():
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


if __name__ == "__main__":
    main()
