"""libmbt.so builds, loads without a GPU, and exports every entry point
include/mbt.h and include/mbt_ws.h declare; calls that need a device fail
with an error code."""
import ctypes
import os
import re

import pytest

from mbtrack_b200 import api
from mbtrack_b200.abi import MbtParams, MbtWsParams

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = "".join(open(os.path.join(ROOT, "include", h)).read() for h in ("mbt.h", "mbt_ws.h"))
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mbt_[a-z_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported(libmbt):
    names = declared_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(libmbt, n), n
        assert n in api.SIGNATURES, "binding lacks %s" % n


def test_params_layout(libmbt):
    assert libmbt.mbt_params_size() == ctypes.sizeof(MbtParams)
    assert libmbt.mbt_ws_params_size() == ctypes.sizeof(MbtWsParams)


def test_no_device_is_an_error_not_a_fallback(libmbt):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    p = MbtParams()
    p.nharm = 4
    p.track_plane[0] = 1
    bucket = (ctypes.c_int * 1)(0)
    npb = (ctypes.c_int * 1)(10)
    ib = (ctypes.c_double * 1)(1e-3)
    h = ctypes.c_void_p()
    rc = libmbt.mbt_create(ctypes.byref(p), 1, ctypes.cast(bucket, ctypes.c_void_p),
                           ctypes.cast(npb, ctypes.c_void_p), ctypes.cast(ib, ctypes.c_void_p),
                           None, None, None, 0, 0, ctypes.byref(h))
    assert rc == -7   # MBT_ERR_NODEVICE
    assert rc != 0 and not h.value
