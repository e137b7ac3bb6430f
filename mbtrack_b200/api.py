"""Python mirror of libmbt's C-ABI (include/mbt.h), used by tests and bench.

Names follow the reference's worker interface: a ``Tracker`` holds every
filled bunch of the ring on one GPU and runs the weak-weak loop of
worker_weakweak.c:259-394 for all of them per call.  There is no CPU path:
loading fails loudly when libmbt.so is missing, and every call that needs
a device fails with MBT_ERR_NODEVICE when there is none.
"""
import ctypes
import os

import numpy as np

from .abi import (MBT_ERR_INVALID, MBT_NOISE_INJECTED, MBT_NOISE_PHILOX, MBT_WRITER_OWN_AMPINV, MbtBeamIon, MbtOutputCfg,
                  MbtParams, MbtState, MbtWsParams)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmbt.so")

_vp = ctypes.c_void_p
_P = ctypes.POINTER
_lib = None

# every symbol include/mbt.h declares, with its ctypes signature
SIGNATURES = {
    "mbt_params_size": (ctypes.c_size_t, []),
    "mbt_config_load": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, _P(MbtParams), _vp, _vp, _vp]),
    "mbt_config_greens": (ctypes.c_int, [ctypes.c_char_p, _P(MbtParams), _vp, _vp, _vp]),
    "mbt_config_error": (ctypes.c_char_p, []),
    "mbt_bunch_current": (ctypes.c_double, [_P(MbtParams), ctypes.c_int, ctypes.c_double]),
    "mbt_rw_first_bin": (ctypes.c_int, [ctypes.c_double, _P(ctypes.c_double), _P(ctypes.c_double)]),
    "mbt_tune_spectra_dev": (ctypes.c_int, [_vp, ctypes.c_long, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp]),
    "mbt_tune_peaks": (ctypes.c_int, [_vp, ctypes.c_long, _vp, _vp, _vp, ctypes.c_int]),
    "mbt_create": (ctypes.c_int, [_P(MbtParams), ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp,
                                  ctypes.c_int, ctypes.c_uint64, _P(_vp)]),
    "mbt_destroy": (ctypes.c_int, [_vp]),
    "mbt_last_error": (ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.c_size_t]),
    "mbt_load_particles": (ctypes.c_int, [_vp, ctypes.c_int, _vp, ctypes.c_int]),
    "mbt_load_all": (ctypes.c_int, [_vp, _vp]),
    "mbt_generate_beam": (ctypes.c_int, [_vp, ctypes.c_uint64]),
    "mbt_get_particles": (ctypes.c_int, [_vp, ctypes.c_int, _vp, ctypes.c_int]),
    "mbt_get_all": (ctypes.c_int, [_vp, _vp]),
    "mbt_prepare": (ctypes.c_int, [_vp, _vp]),
    "mbt_set_deviates": (ctypes.c_int, [_vp, _vp, ctypes.c_long]),
    "mbt_run_turns": (ctypes.c_int, [_vp, ctypes.c_long, _vp]),
    "mbt_run_turns_ampinv": (ctypes.c_int, [_vp, ctypes.c_long, _vp, _vp]),
    "mbt_track": (ctypes.c_int, [_vp, _vp, ctypes.c_long, _vp]),
    "mbt_profile_turns": (ctypes.c_int, [_vp, ctypes.c_long, _vp]),
    "mbt_get_state": (ctypes.c_int, [_vp, _P(MbtState)]),
    "mbt_inject_device_error": (ctypes.c_int, [_vp, ctypes.c_int]),
    "mbt_selftest_bounded_wait": (ctypes.c_int, [ctypes.c_long, _vp]),
    "mbt_get_histograms": (ctypes.c_int, [_vp, ctypes.c_int] + [_vp] * 6),
    "mbt_last_timing": (ctypes.c_int, [_vp, _vp, _vp]),
    "mbt_geometry": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "mbt_set_tiles": (ctypes.c_int, [_vp, _vp]),
    "mbt_autotune": (ctypes.c_int, [_vp, ctypes.c_int, _vp]),
    "mbt_bunch_moments_dev": (ctypes.c_int, [ctypes.c_int, _vp, ctypes.c_double, ctypes.c_double,
                                             ctypes.c_double, ctypes.c_int, _vp, _vp, _vp, _vp]),
    "mbt_bunch_moments_dev_noalloc": (ctypes.c_int, [ctypes.c_int, _vp, ctypes.c_double, ctypes.c_double,
                                                     ctypes.c_double, ctypes.c_int, _vp, _vp, _vp, _vp]),
    "mbt_config_output": (ctypes.c_int, [ctypes.c_char_p, _P(MbtOutputCfg), _vp]),
    "mbt_reference_beam": (ctypes.c_int, [_P(MbtParams), ctypes.c_int, ctypes.c_int, _vp]),
    "mbt_use_device": (ctypes.c_int, [ctypes.c_int]),
    "mbt_get_stats": (ctypes.c_int, [_vp, _vp]),
    "mbt_watch_potentials": (ctypes.c_int, [_vp, ctypes.c_int, _vp]),
    "mbt_get_potentials": (ctypes.c_int, [_vp, ctypes.c_int, _vp]),
    "mbt_writer_open": (ctypes.c_int, [ctypes.c_char_p, _P(MbtParams), _P(MbtOutputCfg), _vp, ctypes.c_int,
                                       _vp, _vp, ctypes.c_int, _P(_vp)]),
    "mbt_writer_wakes": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "mbt_writer_begin": (ctypes.c_int, [_vp, _vp]),
    "mbt_writer_turns": (ctypes.c_int, [_vp, ctypes.c_long, _vp, _vp]),
    "mbt_writer_potentials_due": (ctypes.c_int, [_vp, ctypes.c_long]),
    "mbt_writer_potentials": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_long, _vp, ctypes.c_double,
                                             ctypes.c_double]),
    "mbt_writer_end": (ctypes.c_int, [_vp, _vp]),
    "mbt_writer_distribution": (ctypes.c_int, [_vp, ctypes.c_int, _vp, ctypes.c_int]),
    "mbt_writer_close": (ctypes.c_int, [_vp]),
    "mbt_writer_error": (ctypes.c_char_p, []),
    "mbt_config_beam_ion": (ctypes.c_int, [ctypes.c_char_p, _P(MbtBeamIon)]),
    "mbt_enable_beam_ion": (ctypes.c_int, [_vp, _P(MbtBeamIon)]),
    "mbt_beam_ion_clouds": (ctypes.c_int, [_vp, _vp]),
    "mbt_beam_ion_timing": (ctypes.c_int, [_vp, _vp]),
    "mbt_beam_ion_kernel_times": (ctypes.c_int, [_vp, _vp]),
    "mbt_gauss_field_dev": (ctypes.c_int, [ctypes.c_long, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "mbt_beam_ion_use_mlp": (ctypes.c_int, [_vp, _vp]),
    "mbt_beam_ion_audit": (ctypes.c_int, [_vp, _vp]),
    "mbt_mlp_create": (ctypes.c_int, [ctypes.c_uint64, _P(_vp)]),
    "mbt_mlp_destroy": (ctypes.c_int, [_vp]),
    "mbt_mlp_set_params": (ctypes.c_int, [_vp, _vp]),
    "mbt_mlp_get_params": (ctypes.c_int, [_vp, _vp]),
    "mbt_mlp_forward_dev": (ctypes.c_int, [_vp, ctypes.c_long, _vp, _vp, _vp]),
    "mbt_mlp_gradient": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _vp, _P(ctypes.c_double)]),
    "mbt_mlp_targets_dev": (ctypes.c_int, [ctypes.c_long, _vp, _vp, _vp]),
    "mbt_mlp_field_dev": (ctypes.c_int, [_vp, ctypes.c_long, _vp, _vp, _vp, _vp, _vp, _vp, _P(ctypes.c_long), _vp]),
    "mbt_mlp_train": (ctypes.c_int, [_vp, ctypes.c_long, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                     ctypes.c_uint64, _vp]),
    "mbt_wofz_dev": (ctypes.c_int, [ctypes.c_long, _vp, _vp, _vp, _vp, _vp, _vp]),
    "mbt_be_field_dev": (ctypes.c_int, [ctypes.c_long, _vp, _vp, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_double, _vp, _vp, _vp]),
    "mbt_checkpoint_save": (ctypes.c_int, [_vp, ctypes.c_char_p]),
    "mbt_checkpoint_load": (ctypes.c_int, [_vp, ctypes.c_char_p]),
    "mbt_checkpoint_check": (ctypes.c_int, [ctypes.c_char_p, _P(ctypes.c_long), _P(ctypes.c_int)]),
    # include/mbt_ws.h: the slice model with fast beam-ion interaction
    "mbt_ws_params_size": (ctypes.c_size_t, []),
    "mbt_ws_config_load": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, _P(MbtWsParams), _vp, _vp, _vp]),
    "mbt_ws_slice_beam": (ctypes.c_int, [_P(MbtWsParams), _vp, ctypes.c_int, _vp, _vp, _vp]),
    "mbt_ws_reference_beam": (ctypes.c_int, [_P(MbtWsParams), ctypes.c_int, _vp, _vp]),
    "mbt_ws_create": (ctypes.c_int, [_P(MbtWsParams), ctypes.c_int, _vp, _vp, _vp, _vp, _P(_vp)]),
    "mbt_ws_load_slices": (ctypes.c_int, [_vp, _vp]),
    "mbt_ws_get_slices": (ctypes.c_int, [_vp, _vp]),
    "mbt_ws_run_turns": (ctypes.c_int, [_vp, ctypes.c_long, _vp, _vp, _vp, _vp]),
    "mbt_ws_bunch_fields": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp]),
    "mbt_ws_turn": (ctypes.c_long, [_vp]),
    "mbt_ws_checkpoint_save": (ctypes.c_int, [_vp, ctypes.c_char_p]),
    "mbt_ws_checkpoint_load": (ctypes.c_int, [_vp, ctypes.c_char_p]),
    "mbt_ws_last_ms": (ctypes.c_double, [_vp]),
    "mbt_ws_profile": (ctypes.c_int, [_vp, ctypes.c_long, _vp]),
    "mbt_ws_interp": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _vp, _vp, ctypes.c_int, _vp]),
    "mbt_ws_last_error": (ctypes.c_char_p, [_vp]),
    "mbt_ws_destroy": (None, [_vp]),
    "mbt_ws_writer_open": (ctypes.c_int, [ctypes.c_char_p, _P(MbtWsParams), ctypes.c_int, _vp, ctypes.c_int,
                                          _P(_vp)]),
    "mbt_ws_writer_turns": (ctypes.c_int, [_vp, ctypes.c_long, _vp, _vp, _vp]),
    "mbt_ws_writer_distribution": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int]),
    "mbt_ws_writer_close": (ctypes.c_int, [_vp]),
    "mbt_ws_writer_error": (ctypes.c_char_p, []),
    "mbt_config_bunch_model": (ctypes.c_int, [ctypes.c_char_p]),
}


class MbtError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("libmbt error %d: %s" % (code, msg))
        self.code = code


def lib():
    """Load libmbt.so (built by mbtrack_b200.build); raises when missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libmbt.so not built: run `python -m mbtrack_b200.build` "
                              "(the tracking path has no CPU implementation)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        if L.mbt_params_size() != ctypes.sizeof(MbtParams):
            raise ImportError("mbt_params layout mismatch: C %d bytes, ctypes %d bytes"
                              % (L.mbt_params_size(), ctypes.sizeof(MbtParams)))
        if L.mbt_ws_params_size() != ctypes.sizeof(MbtWsParams):
            raise ImportError("mbt_ws_params layout mismatch: C %d bytes, ctypes %d bytes"
                              % (L.mbt_ws_params_size(), ctypes.sizeof(MbtWsParams)))
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_vp)


def _check(rc, ctx=None):
    if rc != 0:
        buf = ctypes.create_string_buffer(512)
        lib().mbt_last_error(ctx, buf, 512)
        raise MbtError(rc, buf.value.decode(errors="replace"))


class Config:
    """A .conf file read with the reference's semantics (mbt_config_load)."""

    def __init__(self, path, fix_rw_beff=True):
        L = lib()
        self.path = path
        self.params = MbtParams()
        h = 100000
        bucket = np.zeros(h, dtype=np.int32)
        frac = np.zeros(h)
        nb = ctypes.c_int()
        rc = L.mbt_config_load(path.encode(), int(fix_rw_beff), ctypes.byref(self.params),
                               ctypes.byref(nb), _ptr(bucket), _ptr(frac))
        if rc != 0:
            raise MbtError(rc, L.mbt_config_error().decode())
        self.nbunch = nb.value
        self.bucket = bucket[:self.nbunch].copy()
        self.ib_frac = frac[:self.nbunch].copy()
        n = max(self.params.ncell, 1)
        self.Gl, self.Gv, self.Gh = np.zeros(n), np.zeros(n), np.zeros(n)
        rc = L.mbt_config_greens(path.encode(), ctypes.byref(self.params), _ptr(self.Gl),
                                 _ptr(self.Gv), _ptr(self.Gh))
        if rc != 0:
            raise MbtError(rc, L.mbt_config_error().decode())

    def bunch_currents(self):
        L = lib()
        return np.array([L.mbt_bunch_current(ctypes.byref(self.params), self.nbunch, f)
                         for f in self.ib_frac])

    def output(self):
        """(mbt_output_cfg, output bucket numbers) of the file."""
        L = lib()
        o = MbtOutputCfg()
        out = np.zeros(max(self.params.nharm, 1), dtype=np.int32)
        rc = L.mbt_config_output(self.path.encode(), ctypes.byref(o), _ptr(out))
        if rc != 0:
            raise MbtError(rc, L.mbt_config_error().decode())
        return o, out[:o.n_out].copy()

    def beam_ion(self):
        """The [beam_ion] section (MbtBeamIon), or None when absent."""
        L = lib()
        bi = MbtBeamIon()
        rc = L.mbt_config_beam_ion(self.path.encode(), ctypes.byref(bi))
        if rc == 1:
            return None
        if rc != 0:
            raise MbtError(rc, L.mbt_config_error().decode())
        return bi

    def reference_beam(self, np_=None):
        """The reference's initial distribution of every bunch (host),
        a list of [6, np] arrays (mbt_reference_beam)."""
        L = lib()
        n = self.params.np_model if np_ is None else np_
        beams = []
        for kb in self.bucket:
            a = np.zeros((6, n))
            rc = L.mbt_reference_beam(ctypes.byref(self.params), int(kb), n, _ptr(a))
            if rc != 0:
                raise MbtError(rc, "mbt_reference_beam")
            beams.append(a)
        return beams


class Writer:
    """The reference's output files (mbt_writer_*)."""

    def __init__(self, work_path, params, ocfg, bunch_out, bucket, ib, own_ampinv=False):
        L = lib()
        self.params = params.copy()
        self.ocfg = ocfg
        self.bunch_out = np.ascontiguousarray(bunch_out, dtype=np.int32)
        self.bucket = np.ascontiguousarray(bucket, dtype=np.int32)
        self.ib = np.ascontiguousarray(ib, dtype=np.float64)
        self.nb = len(self.bucket)
        h = _vp()
        rc = L.mbt_writer_open(work_path.encode(), ctypes.byref(self.params), ctypes.byref(self.ocfg),
                               _ptr(self.bunch_out), self.nb, _ptr(self.bucket), _ptr(self.ib),
                               MBT_WRITER_OWN_AMPINV if own_ampinv else 0, ctypes.byref(h))
        self._check(rc)
        self.h = h

    def _check(self, rc):
        if rc != 0:
            raise MbtError(rc, lib().mbt_writer_error().decode(errors="replace"))

    def wakes(self, Gl, Gv, Gh):
        g = [np.ascontiguousarray(a, dtype=np.float64) for a in (Gl, Gv, Gh)]
        self._check(lib().mbt_writer_wakes(self.h, *[_ptr(a) for a in g]))

    def begin(self, init_stats):
        a = np.ascontiguousarray(init_stats, dtype=np.float64)
        self._check(lib().mbt_writer_begin(self.h, _ptr(a)))

    def turns(self, stats, ampinv=None):
        st = np.ascontiguousarray(stats, dtype=np.float64)
        ai = None if ampinv is None else np.ascontiguousarray(ampinv, dtype=np.float64)
        self._check(lib().mbt_writer_turns(self.h, st.shape[0], _ptr(st), _ptr(ai)))

    def potentials_due(self, rev):
        return bool(lib().mbt_writer_potentials_due(self.h, rev))

    def potentials(self, ibunch, rev, pot, vrf0, phai0):
        a = np.ascontiguousarray(pot, dtype=np.float64)
        self._check(lib().mbt_writer_potentials(self.h, ibunch, rev, _ptr(a), vrf0, phai0))

    def end(self, end_stats):
        a = np.ascontiguousarray(end_stats, dtype=np.float64)
        self._check(lib().mbt_writer_end(self.h, _ptr(a)))

    def distribution(self, ibunch, soa6):
        a = np.ascontiguousarray(soa6, dtype=np.float64)
        self._check(lib().mbt_writer_distribution(self.h, ibunch, _ptr(a), a.size // 6))

    def close(self):
        if getattr(self, "h", None):
            lib().mbt_writer_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Tracker:
    """One tracking context (mbt_ctx) holding every filled bunch."""

    def __init__(self, params, bucket, np_, ib, Gl=None, Gv=None, Gh=None,
                 noise=MBT_NOISE_PHILOX, seed=0):
        L = lib()
        self.params = params.copy()
        self.bucket = np.ascontiguousarray(bucket, dtype=np.int32)
        self.np = np.ascontiguousarray(np_, dtype=np.int32)
        self.ib = np.ascontiguousarray(ib, dtype=np.float64)
        self.nb = len(self.bucket)
        g = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (Gl, Gv, Gh)]
        self._g = g
        h = _vp()
        rc = L.mbt_create(ctypes.byref(self.params), self.nb, _ptr(self.bucket), _ptr(self.np),
                          _ptr(self.ib), _ptr(g[0]), _ptr(g[1]), _ptr(g[2]), noise, seed,
                          ctypes.byref(h))
        _check(rc, None)
        self.h = h

    @classmethod
    def from_config(cls, cfg, np_per_bunch=None, noise=MBT_NOISE_PHILOX, seed=0):
        n = np.full(cfg.nbunch, cfg.params.np_model if np_per_bunch is None else np_per_bunch)
        return cls(cfg.params, cfg.bucket, n, cfg.bunch_currents(), cfg.Gl, cfg.Gv, cfg.Gh,
                   noise=noise, seed=seed)

    def checkpoint_save(self, path):
        """mbt_checkpoint_save: the state that carries into the next turn."""
        _check(lib().mbt_checkpoint_save(self.h, path.encode()), self.h)

    def checkpoint_load(self, path):
        """mbt_checkpoint_load into this prepared context."""
        _check(lib().mbt_checkpoint_load(self.h, path.encode()), self.h)

    def close(self):
        if getattr(self, "h", None):
            lib().mbt_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load_particles(self, ib, soa6):
        a = np.ascontiguousarray(soa6, dtype=np.float64).ravel()
        if a.size % 6:
            raise ValueError("a soa6 buffer holds 6 arrays of equal length")
        _check(lib().mbt_load_particles(self.h, ib, _ptr(a), a.size // 6), self.h)

    def load_all(self, soa6_all):
        a = np.ascontiguousarray(soa6_all, dtype=np.float64)
        assert a.size == 6 * int(self.np.sum())
        _check(lib().mbt_load_all(self.h, _ptr(a)), self.h)

    def generate_beam(self, seed):
        _check(lib().mbt_generate_beam(self.h, seed), self.h)

    def get_particles(self, ib):
        a = np.empty(6 * int(self.np[ib]))
        _check(lib().mbt_get_particles(self.h, ib, _ptr(a), int(self.np[ib])), self.h)
        return a.reshape(6, int(self.np[ib]))

    def get_all(self):
        a = np.empty(6 * int(self.np.sum()))
        _check(lib().mbt_get_all(self.h, _ptr(a)), self.h)
        return a

    def get_stats(self):
        """Statistics of the current coordinates (pending RW kick included)."""
        s = np.zeros(12 * self.nb)
        _check(lib().mbt_get_stats(self.h, _ptr(s)), self.h)
        return s.reshape(self.nb, 12)

    def enable_beam_ion(self, bi):
        _check(lib().mbt_enable_beam_ion(self.h, ctypes.byref(bi)), self.h)
        self.bi = bi

    def beam_ion_clouds(self):
        a = np.zeros(self.bi.n_ip * self.nb * 5)
        _check(lib().mbt_beam_ion_clouds(self.h, _ptr(a)), self.h)
        return a.reshape(self.bi.n_ip, self.nb, 5)

    def use_mlp(self, mlp):
        _check(lib().mbt_beam_ion_use_mlp(self.h, mlp.h), self.h)
        self._mlp = mlp

    def beam_ion_audit(self):
        """(audited, max rel. error, rms rel. error, fallbacks, failures)."""
        a = np.zeros(5)
        _check(lib().mbt_beam_ion_audit(self.h, _ptr(a)), self.h)
        return a

    def beam_ion_timing(self):
        v = ctypes.c_double()
        _check(lib().mbt_beam_ion_timing(self.h, ctypes.byref(v)), self.h)
        return v.value

    def beam_ion_kernel_times(self):
        """ms per turn of (frames, ions, clouds, electron kicks), last profile."""
        v = np.zeros(4)
        _check(lib().mbt_beam_ion_kernel_times(self.h, _ptr(v)), self.h)
        return v

    def watch_potentials(self, bunches):
        b = np.ascontiguousarray(bunches, dtype=np.int32)
        _check(lib().mbt_watch_potentials(self.h, len(b), _ptr(b)), self.h)

    def potentials(self, ib):
        """7 x ncell potential terms of the next turn (mbt_get_potentials)."""
        a = np.zeros(7 * self.params.ncell)
        _check(lib().mbt_get_potentials(self.h, ib, _ptr(a)), self.h)
        return a.reshape(7, self.params.ncell)

    def prepare(self):
        s = np.zeros(12 * self.nb)
        _check(lib().mbt_prepare(self.h, _ptr(s)), self.h)
        return s.reshape(self.nb, 12)

    def set_deviates(self, dev, nturns):
        d = np.ascontiguousarray(dev, dtype=np.float32).ravel()
        per = 1 + 2 * (self.params.track_plane[2] != 0) + 2 * (self.params.track_plane[1] != 0)
        if d.size < nturns * per * int(self.np.sum()):
            raise ValueError("%d deviates given, %d turns need %d"
                             % (d.size, nturns, nturns * per * int(self.np.sum())))
        _check(lib().mbt_set_deviates(self.h, _ptr(d), nturns), self.h)

    def run(self, nturns, stats=True):
        s = np.zeros(nturns * self.nb * 12) if stats else None
        _check(lib().mbt_run_turns(self.h, nturns, _ptr(s)), self.h)
        return None if s is None else s.reshape(nturns, self.nb, 12)

    def run_ampinv(self, nturns):
        """Statistics and amplitude invariants of every turn."""
        s = np.zeros(nturns * self.nb * 12)
        ai = np.zeros(nturns * self.nb * 6)
        _check(lib().mbt_run_turns_ampinv(self.h, nturns, _ptr(s), _ptr(ai)), self.h)
        return s.reshape(nturns, self.nb, 12), ai.reshape(nturns, self.nb, 6)

    def track(self, particles, nturns, stats=None):
        if particles.dtype != np.float64 or not particles.flags.c_contiguous or \
                particles.size != 6 * int(self.np.sum()):
            raise ValueError("particles must be a contiguous float64 buffer of 6 * sum(np)")
        if stats is not None and (stats.dtype != np.float64 or stats.size < nturns * self.nb * 12):
            raise ValueError("stats must hold nturns * nbunch * 12 doubles")
        _check(lib().mbt_track(self.h, _ptr(particles), nturns, _ptr(stats)), self.h)

    def profile(self, nturns):
        out = np.zeros(4)
        _check(lib().mbt_profile_turns(self.h, nturns, _ptr(out)), self.h)
        return out

    def inject_device_error(self, bits):
        """mbt_inject_device_error: set bits of the sticky device error word."""
        _check(lib().mbt_inject_device_error(self.h, bits), self.h)

    def state(self):
        st = MbtState()
        _check(lib().mbt_get_state(self.h, ctypes.byref(st)), self.h)
        return st

    def histograms(self, ib):
        n = self.params.ncell
        arr = [np.zeros(n) for _ in range(6)]
        _check(lib().mbt_get_histograms(self.h, ib, *[_ptr(a) for a in arr]), self.h)
        return arr

    def set_tiles(self, tiles):
        t = np.ascontiguousarray(tiles, dtype=np.int32)
        _check(lib().mbt_set_tiles(self.h, _ptr(t)), self.h)

    def autotune(self, trial_turns=10):
        t = np.zeros(3, dtype=np.int32)
        _check(lib().mbt_autotune(self.h, trial_turns, _ptr(t)), self.h)
        return t

    def timing(self):
        out = np.zeros(4)
        nl = ctypes.c_int()
        _check(lib().mbt_last_timing(self.h, _ptr(out), ctypes.byref(nl)), self.h)
        return out, nl.value

    def geometry(self):
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(lib().mbt_geometry(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)), self.h)
        return a.value, b.value, c.value


def rw_first_bin(u):
    """(longitudinal, transverse) first-bin values of the short-range
    resistive wall for a bin of u s0 (mbt_rw_first_bin)."""
    a, b = ctypes.c_double(), ctypes.c_double()
    if lib().mbt_rw_first_bin(float(u), ctypes.byref(a), ctypes.byref(b)) != 0:
        raise MbtError(MBT_ERR_INVALID, "bin of %g s0 is narrower than 19.8 s0" % u)
    return a.value, b.value


def tune_spectra_dev(x_ptr, ld, nseries, nturn, plane, spec_ptr, stream=None):
    """Normalised tune spectra of device centroid histories (mbt_tune_spectra_dev)."""
    _gchk(lib().mbt_tune_spectra_dev(x_ptr, ld, nseries, nturn, plane, spec_ptr, stream))


def tune_peaks(spec, nrev, max_peaks=10):
    """(values, amplitudes, cases) of the peaks of one normalised spectrum
    (mbt_tune_peaks)."""
    s = np.ascontiguousarray(spec, dtype=np.float64)
    v = np.zeros(max_peaks)
    a = np.zeros(max_peaks)
    c = np.zeros(max_peaks, dtype=np.int32)
    n = lib().mbt_tune_peaks(_ptr(s), nrev, _ptr(v), _ptr(a), _ptr(c), max_peaks)
    if n < 0:
        raise MbtError(n, "tune peaks: bad argument")
    return v[:n], a[:n], c[:n]


def wofz_dev(x_ptr, y_ptr, re_ptr, im_ptr, n, flag_ptr=None, stream=None):
    """w(z) on device buffers (raw pointers, e.g. torch .data_ptr())."""
    _check(lib().mbt_wofz_dev(n, x_ptr, y_ptr, re_ptr, im_ptr, flag_ptr, stream))


def be_field_dev(dx_ptr, dy_ptr, n, sgm_xx_mm, sgm_zz_mm, factdq, ex_ptr, ey_ptr, stream=None):
    _check(lib().mbt_be_field_dev(n, dx_ptr, dy_ptr, sgm_xx_mm, sgm_zz_mm, factdq, ex_ptr, ey_ptr, stream))


def bunch_moments_dev(np_, coord_ptr, sigma_tau, nsigma, dT, ncell, track_plane, hist_ptr=None, stream=None):
    """Statistics (12 values, mbt.h order) of one bunch on the device; the
    in-range histograms go to hist_ptr (3 x ncell doubles, device)."""
    st = np.zeros(12)
    tp = np.ascontiguousarray(track_plane, dtype=np.int32)
    _check(lib().mbt_bunch_moments_dev(np_, coord_ptr, sigma_tau, nsigma, dT, ncell, _ptr(tp), _ptr(st),
                                       hist_ptr, stream))
    return st


def bunch_moments_dev_noalloc(np_, coord_ptr, sigma_tau, nsigma, dT, ncell, track_plane, hist_ptr=None,
                              stream=None):
    """As bunch_moments_dev, through the entry point that allocates nothing
    (its scratch is a fixed device array inside libmbt)."""
    st = np.zeros(12)
    tp = np.ascontiguousarray(track_plane, dtype=np.int32)
    _check(lib().mbt_bunch_moments_dev_noalloc(np_, coord_ptr, sigma_tau, nsigma, dT, ncell, _ptr(tp),
                                               _ptr(st), hist_ptr, stream))
    return st


MLP_NPARAM = 33794


def _gchk(rc):
    if rc != 0:
        buf = ctypes.create_string_buffer(512)
        lib().mbt_last_error(None, buf, 512)
        raise MbtError(rc, buf.value.decode(errors="replace"))


# Training settings of the learned field for the beam-ion runs (bench.py and
# the tests of the field-error and growth-rate tolerances): 1e7 seeded
# samples labelled by the Faddeeva field, minibatches of 8192, Adam at 2e-3
# with cosine decay.
MLP_TRAIN = {"nsamples": 10_000_000, "batch": 8192, "steps": 20000, "lr": 2e-3}


class Mlp:
    """The learned field network (mbt_mlp_*).  Device arrays are passed as
    integer addresses (e.g. torch tensors' data_ptr())."""

    def __init__(self, seed=1):
        h = _vp()
        _gchk(lib().mbt_mlp_create(seed, ctypes.byref(h)))
        self.h = h

    def params(self):
        a = np.zeros(MLP_NPARAM, dtype=np.float32)
        _gchk(lib().mbt_mlp_get_params(self.h, _ptr(a)))
        return a

    def set_params(self, p):
        a = np.ascontiguousarray(p, dtype=np.float32)
        assert a.size == MLP_NPARAM
        _gchk(lib().mbt_mlp_set_params(self.h, _ptr(a)))

    def forward_dev(self, n, abr_ptr, out_ptr):
        _gchk(lib().mbt_mlp_forward_dev(self.h, n, abr_ptr, out_ptr, None))

    def gradient_dev(self, n, abr_ptr, tgt_ptr):
        g = np.zeros(MLP_NPARAM, dtype=np.float32)
        loss = ctypes.c_double()
        _gchk(lib().mbt_mlp_gradient(self.h, n, abr_ptr, tgt_ptr, _ptr(g), ctypes.byref(loss)))
        return g, loss.value

    def field_dev(self, n, dx_ptr, dy_ptr, sx_ptr, sy_ptr, gx_ptr, gy_ptr):
        """mbt_mlp_field_dev: the learned field at n points; returns the
        number of points outside the network's domain."""
        fb = ctypes.c_long()
        _gchk(lib().mbt_mlp_field_dev(self.h, n, dx_ptr, dy_ptr, sx_ptr, sy_ptr, gx_ptr, gy_ptr, ctypes.byref(fb),
                                      None))
        return fb.value

    def train(self, nsamples, batch, steps, lr, seed):
        hist = np.zeros(steps, dtype=np.float32)
        _gchk(lib().mbt_mlp_train(self.h, nsamples, batch, steps, lr, seed, _ptr(hist)))
        return hist

    def close(self):
        if getattr(self, "h", None):
            lib().mbt_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def mlp_targets_dev(n, abr_ptr, tgt_ptr):
    _gchk(lib().mbt_mlp_targets_dev(n, abr_ptr, tgt_ptr, None))


class SliceModel:
    """The slice model (BunchModel = STRONG) with fast beam-ion interaction
    on one GPU (include/mbt_ws.h): manager_weakstrong / worker_weakstrong
    of the reference for every filled bunch at once."""

    def __init__(self, w, bucket, ibunch, npop, nofe):
        L = lib()
        self.w = w
        self.nb = len(bucket)
        self.S = w.slices
        self.nion = self.S * w.ngrid * w.ngrid
        self.nharm = w.base.nharm
        keep = [np.ascontiguousarray(bucket, dtype=np.int32), np.ascontiguousarray(ibunch, dtype=np.float64),
                np.ascontiguousarray(npop, dtype=np.int32), np.ascontiguousarray(nofe, dtype=np.int32)]
        h = _vp()
        rc = L.mbt_ws_create(ctypes.byref(w), self.nb, *[_ptr(a) for a in keep], ctypes.byref(h))
        if rc != 0:
            raise MbtError(rc, L.mbt_ws_last_error(None).decode(errors="replace"))
        self.h = h

    @staticmethod
    def config(path, fix_rw_beff=True):
        """(mbt_ws_params, bucket, ib_frac) of a BunchModel = STRONG .conf."""
        L = lib()
        w = MbtWsParams()
        nb = ctypes.c_int()
        cap = 4096
        bucket = np.zeros(cap, np.int32)
        frac = np.zeros(cap)
        rc = L.mbt_ws_config_load(path.encode(), int(fix_rw_beff), ctypes.byref(w), ctypes.byref(nb), _ptr(bucket),
                                  _ptr(frac))
        if rc != 0:
            raise MbtError(rc, L.mbt_config_error().decode(errors="replace"))
        return w, bucket[:nb.value].copy(), frac[:nb.value].copy()

    @staticmethod
    def slice_beam(w, soa6):
        """mbt_ws_slice_beam: (npop[S], nofe[S, G, G], cm4[4, S])."""
        soa6 = np.ascontiguousarray(soa6, dtype=np.float64)
        S, G = w.slices, w.ngrid
        npop = np.zeros(S, np.int32)
        nofe = np.zeros((S, G, G), np.int32)
        cm4 = np.zeros((4, S))
        rc = lib().mbt_ws_slice_beam(ctypes.byref(w), _ptr(soa6), soa6.shape[1], _ptr(npop), _ptr(nofe), _ptr(cm4))
        if rc != 0:
            raise MbtError(rc, "mbt_ws_slice_beam failed")
        return npop, nofe, cm4

    @staticmethod
    def reference_beam(w, nbunch):
        """mbt_ws_reference_beam: (soa6[6, np], off4[nbunch, 4])."""
        soa6 = np.zeros((6, w.np))
        off4 = np.zeros((nbunch, 4))
        rc = lib().mbt_ws_reference_beam(ctypes.byref(w), nbunch, _ptr(soa6), _ptr(off4))
        if rc != 0:
            raise MbtError(rc, "mbt_ws_reference_beam failed")
        return soa6, off4

    @staticmethod
    def initial_slices(w, cm4, off4):
        """The manager's starting slices (generate_initial_general_
        distribution2): cm4 plus each bunch's offsets, xtau/xeps zero."""
        nb = off4.shape[0]
        s = np.zeros((nb, 6, w.slices))
        for k in range(4):
            s[:, 2 + k, :] = cm4[k][None, :] + off4[:, k][:, None]
        return s

    def _chk(self, rc):
        if rc != 0:
            raise MbtError(rc, lib().mbt_ws_last_error(self.h).decode(errors="replace"))

    def load_slices(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        assert a.shape == (self.nb, 6, self.S)
        self._chk(lib().mbt_ws_load_slices(self.h, _ptr(a)))

    def slices(self):
        a = np.zeros((self.nb, 6, self.S))
        self._chk(lib().mbt_ws_get_slices(self.h, _ptr(a)))
        return a

    @property
    def turn(self):
        return lib().mbt_ws_turn(self.h)

    def run(self, nturns, outputs=True):
        """Run nturns turns; returns (cm, ion, zcm, stats) as mbt_ws_run_turns
        fills them (None each when outputs is False)."""
        if not outputs:
            self._chk(lib().mbt_ws_run_turns(self.h, nturns, None, None, None, None))
            return None, None, None, None
        t0 = self.turn
        nmon = sum(1 for r in range(t0, t0 + nturns) if r % self.w.base.nrev_mon == 0)
        cm = np.zeros((nturns, self.nb, 6))
        ion = np.zeros((nturns, self.nb, 2))
        zcm = np.zeros((nturns, self.nharm))
        st = np.zeros((max(nmon, 1), self.nb, 18))
        self._chk(lib().mbt_ws_run_turns(self.h, nturns, _ptr(cm), _ptr(ion), _ptr(zcm), _ptr(st)))
        return cm, ion, zcm, st[:nmon]

    def checkpoint_save(self, path):
        self._chk(lib().mbt_ws_checkpoint_save(self.h, path.encode()))

    def checkpoint_load(self, path):
        self._chk(lib().mbt_ws_checkpoint_load(self.h, path.encode()))

    def last_ms(self):
        """Device time [ms] of the last run."""
        return lib().mbt_ws_last_ms(self.h)

    def profile(self, nturns):
        """Mean device ms per turn of (bunch step, optic + RW, ion train, kicks)."""
        ms = np.zeros(4)
        self._chk(lib().mbt_ws_profile(self.h, nturns, _ptr(ms)))
        return ms

    def interp(self, ib, icell, x, y):
        """The device's grid interpolation on bunch ib's last field grid."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.ascontiguousarray(y, dtype=np.float64)
        out = np.zeros((x.size, 2))
        self._chk(lib().mbt_ws_interp(self.h, ib, icell, _ptr(x), _ptr(y), x.size, _ptr(out)))
        return out

    def bunch_fields(self, ib):
        e = np.zeros((self.nion, 2))
        ions = np.zeros((5, self.nion))
        self._chk(lib().mbt_ws_bunch_fields(self.h, ib, _ptr(e), _ptr(ions)))
        return e, ions

    def close(self):
        if getattr(self, "h", None):
            lib().mbt_ws_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SliceWriter:
    """The slice-model manager's output files (mbt_ws_writer_*)."""

    def __init__(self, work_path, w, bucket, own_ampinv=False):
        L = lib()
        self.w = w
        self._bucket = np.ascontiguousarray(bucket, dtype=np.int32)
        h = _vp()
        rc = L.mbt_ws_writer_open(work_path.encode(), ctypes.byref(w), len(bucket), _ptr(self._bucket),
                                  MBT_WRITER_OWN_AMPINV if own_ampinv else 0, ctypes.byref(h))
        if rc != 0:
            raise MbtError(rc, L.mbt_ws_writer_error().decode(errors="replace"))
        self.h = h

    def _chk(self, rc):
        if rc != 0:
            raise MbtError(rc, lib().mbt_ws_writer_error().decode(errors="replace"))

    def turns(self, ion, zcm, stats):
        ion = np.ascontiguousarray(ion, dtype=np.float64)
        zcm = np.ascontiguousarray(zcm, dtype=np.float64)
        stats = None if stats is None or len(stats) == 0 else np.ascontiguousarray(stats, dtype=np.float64)
        self._chk(lib().mbt_ws_writer_turns(self.h, zcm.shape[0], _ptr(ion), _ptr(zcm), _ptr(stats)))

    def distribution(self, paths, soa6):
        arr = (ctypes.c_char_p * 3)(*[p.encode() for p in paths])
        soa6 = np.ascontiguousarray(soa6, dtype=np.float64)
        self._chk(lib().mbt_ws_writer_distribution(self.h, ctypes.cast(arr, _vp), _ptr(soa6), soa6.shape[1]))

    def close(self):
        if getattr(self, "h", None):
            h, self.h = self.h, None
            self._chk(lib().mbt_ws_writer_close(h))


def checkpoint_check(path):
    """mbt_checkpoint_check: (turn, nbunch) of a checkpoint file, checked on
    the host (structure and checksum); raises MbtError for a bad file."""
    t = ctypes.c_long()
    n = ctypes.c_int()
    rc = lib().mbt_checkpoint_check(path.encode(), ctypes.byref(t), ctypes.byref(n))
    if rc != 0:
        _check(rc, None)
    return t.value, n.value
