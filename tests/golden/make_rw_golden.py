"""Generates tests/golden/rw_first_bin.npz: the first-bin values of the
reference's short-range resistive wall (RW_table_LON / RW_table_TRANS,
rw_table.c:310-391) at a spread of bin widths u (in s0), by calling the
reference's own compiled functions (oracle/_ref/libmbtref.so).

    python tests/golden/make_rw_golden.py
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import binding  # noqa: E402


def main():
    so = binding.build_reference()
    ref = ctypes.CDLL(so or binding.REF_SO)
    for f in (ref.RW_table_LON, ref.RW_table_TRANS):
        f.argtypes = [ctypes.c_double, ctypes.POINTER(ctypes.c_double)]
        f.restype = ctypes.c_int
    rng = np.random.default_rng(7)
    u = np.concatenate([[19.8, 20.0, 20.3, 50.0, 99.5, 500.0, 1999.0, 2400.0],
                        np.exp(rng.uniform(np.log(19.8), np.log(2000.0), 56))])
    lon = np.zeros_like(u)
    trans = np.zeros_like(u)
    for i, x in enumerate(u):
        a, b = ctypes.c_double(), ctypes.c_double()
        assert ref.RW_table_LON(float(x), a) == 1 and ref.RW_table_TRANS(float(x), b) == 1
        lon[i], trans[i] = a.value, b.value
    out = os.path.join(HERE, "rw_first_bin.npz")
    np.savez_compressed(out, u=u, lon=lon, trans=trans)
    print(out, len(u), "values")


if __name__ == "__main__":
    main()
