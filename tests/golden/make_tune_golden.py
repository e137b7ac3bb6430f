"""Generates tests/golden/tune_peaks.npz: the reference's coherent tune
analysis (tune.c, compiled into oracle/_ref/libmbtref.so with the GSL
routine it calls restated in oracle/gsl_fft_stub.c) on seeded inputs:

* identify_tunepeaks (tune.c:383-480) on normalised spectra with planted
  single-bin peaks, plateaus and noise;
* the LON branch of get_tunepeaks_coherent (tune.c:175-233) on centroid
  histories made of damped sinusoids and noise.

    python tests/golden/make_tune_golden.py
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import binding  # noqa: E402

NSPEC, NREV = 40, 256
NHIST, NT = 12, 9


def spectra(rng):
    out = np.zeros((NSPEC, NREV // 2 + 1))
    for s in range(NSPEC):
        c = 0.05 * rng.random(NREV // 2 + 1)
        for _ in range(rng.integers(1, 6)):
            j = int(rng.integers(2, NREV // 2 - 3))
            w = int(rng.integers(0, 4))            # 0: one bin, else a plateau
            c[j:j + w + 1] = rng.uniform(0.3, 1.0)
        c[0] = 0.0
        out[s] = c / c.max()
    return out


def histories(rng):
    n = 1 << NT
    t = np.arange(n)
    out = np.zeros((NHIST, n))
    for h in range(NHIST):
        x = 0.01 * rng.normal(size=n)
        for _ in range(rng.integers(1, 4)):
            f = rng.uniform(0.003, 0.49)
            out_amp = rng.uniform(0.2, 1.0)
            x += out_amp * np.exp(-t / rng.uniform(300, 5000)) * np.cos(2 * np.pi * f * t + rng.uniform(0, 6.3))
        out[h] = x + rng.uniform(-0.5, 0.5)
    return out


def run(fn, arr, *args):
    v, a = np.zeros(10), np.zeros(10)
    txt = ctypes.create_string_buffer(1 << 16)
    p = lambda x: x.ctypes.data_as(ctypes.c_void_p)
    n = fn(p(np.ascontiguousarray(arr)), *args, p(v), p(a), 10, txt, 1 << 16)
    return n, v, a, txt.value.decode()


def main():
    lib = ctypes.CDLL(binding.build_reference() or binding.REF_SO)
    lib.refh_tune_identify.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_int, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
    lib.refh_tune_lon.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                  ctypes.c_char_p, ctypes.c_int]
    rng = np.random.default_rng(2024)
    spec = spectra(rng)
    hist = histories(rng)
    sn, sv, sa, st = [], [], [], []
    for s in spec:
        n, v, a, txt = run(lib.refh_tune_identify, s, NREV, 1)
        sn.append(n); sv.append(v); sa.append(a); st.append(txt)
    hn, hv, ha = [], [], []
    for h in hist:
        n, v, a, _ = run(lib.refh_tune_lon, h, NT)
        hn.append(n); hv.append(v); ha.append(a)
    out = os.path.join(HERE, "tune_peaks.npz")
    np.savez_compressed(out, spec=spec, spec_n=np.array(sn), spec_value=np.array(sv), spec_ampli=np.array(sa),
                        spec_text=np.array(st), hist=hist, hist_n=np.array(hn), hist_value=np.array(hv),
                        hist_ampli=np.array(ha), nrev=NREV, nt=NT)
    print(out, "peaks per spectrum", sn, "per history", hn)


if __name__ == "__main__":
    main()
