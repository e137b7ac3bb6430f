"""Writes uneven_fill.txt, the fill pattern of the uneven batched
configuration, in the reference's fill-file format (e_beam_fileread,
input.c:1445-1512: one `bucket ratio out` line per bucket).

416 buckets: three trains (107, 107, 106 bunches) separated by three gaps of
32 empty buckets, plus a 5 nC camshaft bunch in the middle of the last gap.
Train bunch charges are lognormal with median 0.5 nC and sigma_log 0.3
(numpy seed 20261203).  The ratio column is the charge in nC.  The printed
ring current is sum(q) / T0 for T0 = 416 / 352 MHz.
"""
import os

import numpy as np

H = 416
TRAINS = [(0, 107), (139, 107), (278, 106)]
CAMSHAFT = 400


def charges():
    rng = np.random.default_rng(20261203)
    q = np.zeros(H)
    for start, n in TRAINS:
        q[start:start + n] = 0.5 * np.exp(0.3 * rng.standard_normal(n))
    q[CAMSHAFT] = 5.0
    return q


def main(path=None):
    q = charges()
    path = path or os.path.join(os.path.dirname(os.path.abspath(__file__)), "uneven_fill.txt")
    with open(path, "w") as f:
        for k in range(H):
            out = 1 if k in (0, 50, 139, CAMSHAFT) else 0
            f.write("%d %.10f %d\n" % (k, q[k], out))
    t0 = H / 352.0e6
    print("filled", int((q > 0).sum()), "Iring[mA] %.6f" % (q.sum() * 1e-9 / t0 * 1e3))
    return path


if __name__ == "__main__":
    main()
