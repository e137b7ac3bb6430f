"""Generates tests/golden/writer_<case>.npz: the output files of a whole
reference run, written by the reference's own printing functions through
oracle/ref_harness.c (refh_run_files), together with the statistics stream
they were printed from.

    python tests/golden/make_writer_golden.py

Each fixture holds the text of every file the reference's manager and
output workers write (mean_bunch_*.dat, ampinv_*.dat, bunchbybunch_*.dat,
potentials_bunch_*.dat, wakes.dat, dipoles_history.dat, the distribution
files), the initial, per-turn and end statistics, the amplitude invariants,
the RF voltage and phase at the start of every turn, and the end
coordinates of the first output bunch.  The writer tests feed that stream to
libmbt's writer; the GPU test runs mbtrack-gpu on the same configuration.
"""
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.binding import Reference  # noqa: E402
from tests.util import WRITER_CASES, writer_conf  # noqa: E402


def run_case(case):
    tmp = tempfile.mkdtemp()
    work = os.path.join(tmp, "work")
    os.makedirs(work)
    conf = writer_conf(tmp, case)
    cwd = os.getcwd()
    os.chdir(work)            # the distribution files are relative names
    try:
        R = Reference(conf, workdir=work)
        st0 = R.prepare()
        st, ai, vp, end = R.run_files()
        info = R.output_info()
        first = [i for i in range(R.nb) if R.bucket[i] in set(info["bunch_out"].tolist())]
        final = R.get_particles(first[0]).reshape(6, -1) if first else np.zeros((6, 0))
    finally:
        os.chdir(cwd)
    files = {f: open(os.path.join(work, f)).read() for f in sorted(os.listdir(work))}
    out = os.path.join(HERE, "writer_%s.npz" % case)
    np.savez_compressed(out, init_stats=st0, stats=st, ampinv=ai, vrfphi=vp, end_stats=end,
                        final=final, bucket=R.bucket, ib=R.ib, files=json.dumps(files),
                        bunch_out=info["bunch_out"])
    print(case, "->", out, os.path.getsize(out), "bytes,", len(files), "files")


if __name__ == "__main__":
    for c in sys.argv[1:] or list(WRITER_CASES):
        run_case(c)
