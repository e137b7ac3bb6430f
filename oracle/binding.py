"""ctypes bindings of the oracle (liboracle.so, the C restatement) and of the
reference harness (_ref/libmbtref.so, the reference's own sources).

TEST INFRASTRUCTURE ONLY: used by tests/, smoke() and bench.py's CPU
baseline as the checker, never by the product.
"""
import ctypes
import os
import re
import shutil
import subprocess
import tempfile

import numpy as np

from mbtrack_b200.abi import MbtParams, MbtWsParams

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libmbtref.so")
# the reference tree this library is built from (present in the build
# container only); MBT_REFERENCE_DIR overrides the default location
REFERENCE_DIR = os.environ.get("MBT_REFERENCE_DIR", "/root/reference")

_vp = ctypes.c_void_p
_P = ctypes.POINTER


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_vp)


def build_oracle(force=False):
    """Compile liboracle.so (plain C, gcc) if missing."""
    if force or not os.path.exists(ORACLE_SO):
        subprocess.check_call(["make", "-s", "-C", HERE, "liboracle.so"])
    return ORACLE_SO


def reference_available():
    return os.path.isdir(os.path.join(REFERENCE_DIR, "src"))


def build_reference(force=False):
    """Compile the reference's own sources into _ref/libmbtref.so.

    Needs the reference tree (present in the build container only); on a
    machine without it an already built library is used as is."""
    if os.path.exists(REF_SO) and not force:
        return REF_SO
    if not reference_available():
        return None
    subprocess.check_call(["make", "-s", "-C", HERE, "ref", "REF=" + REFERENCE_DIR])
    return REF_SO


def conf_with(src, dst, **overrides):
    """Copy a .conf file replacing `key = value` lines (each key once)."""
    text = open(src).read()
    for k, v in overrides.items():
        text, n = re.subn(r"(?m)^(\s*%s\s*=).*$" % re.escape(k), r"\g<1> %s" % v, text)
        if n != 1:
            raise KeyError("%s appears %d times in %s" % (k, n, src))
    with open(dst, "w") as f:
        f.write(text)
    return dst


def beam_ion_section(conf):
    """The [beam_ion] section of a .conf file (an MbtBeamIon), read here
    for the C restatement with the defaults and units that libmbt's
    mbt_config_beam_ion documents (pressure in nTorr, cross-section in Mb);
    None when the file has no such section."""
    from mbtrack_b200.abi import MbtBeamIon
    section, vals, seen = None, {}, False
    for line in open(conf):
        t = line.split("#", 1)[0].strip()
        if t.startswith("[") and t.endswith("]"):
            section = t[1:-1].strip()
            seen = seen or section == "beam_ion"
        elif section == "beam_ion" and "=" in t:
            k, v = t.split("=", 1)
            vals[k.strip()] = v.strip()
    if not seen:
        return None
    bi = MbtBeamIon()
    bi.n_ip = int(vals.get("n_ip", 1))
    bi.ions_per_passage = int(vals.get("ions_per_passage", 1000))
    bi.gas_A = float(vals.get("gas_A", 28.0))
    bi.pressure = float(vals.get("pressure_nTorr", 1.0)) * 1e-9
    bi.sigma_ion = float(vals.get("sigma_ion_Mb", 1.78)) * 1e-22
    bi.seed = int(vals.get("seed", 1)) & 0xFFFFFFFF
    bi.surrogate = int(vals.get("surrogate", 0))
    bi.audit_fraction = float(vals.get("audit_fraction", 0.01))
    return bi


class Oracle:
    """The C restatement (mbt_oracle.c)."""

    def __init__(self, params, bucket, np_, ib, Gl=None, Gv=None, Gh=None):
        self.lib = ctypes.CDLL(build_oracle())
        L = self.lib
        L.orc_create.restype = _vp
        L.orc_create.argtypes = [_P(MbtParams), ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp]
        L.orc_run.restype = ctypes.c_long
        L.orc_run.argtypes = [_vp, ctypes.c_long, _vp, _vp, _vp, ctypes.c_long]
        L.orc_deviates_per_turn.restype = ctypes.c_long
        L.orc_deviates_per_turn.argtypes = [_vp]
        for f in ("orc_generate_beam", "orc_prepare", "orc_set_particles", "orc_get_particles"):
            getattr(L, f).restype = ctypes.c_int
        L.orc_generate_beam.argtypes = [_vp]
        L.orc_prepare.argtypes = [_vp, _vp]
        L.orc_set_particles.argtypes = [_vp, ctypes.c_int, _vp]
        L.orc_get_particles.argtypes = [_vp, ctypes.c_int, _vp]
        L.orc_state.argtypes = [_vp, ctypes.c_int, _vp, _vp]
        L.orc_trash.argtypes = [_vp, ctypes.c_int, _vp, _vp]
        L.orc_histograms.argtypes = [_vp, ctypes.c_int] + [_vp] * 6
        L.orc_destroy.argtypes = [_vp]
        L.orc_set_range.argtypes = [_vp, ctypes.c_int, ctypes.c_int]
        self.p = params.copy()
        self.bucket = np.ascontiguousarray(bucket, dtype=np.int32)
        self.np = np.ascontiguousarray(np_, dtype=np.int32)
        self.ib = np.ascontiguousarray(ib, dtype=np.float64)
        self.nb = len(self.bucket)
        g = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (Gl, Gv, Gh)]
        self._g = g
        self.h = L.orc_create(ctypes.byref(self.p), self.nb, _ptr(self.bucket), _ptr(self.np),
                              _ptr(self.ib), _ptr(g[0]), _ptr(g[1]), _ptr(g[2]))
        if not self.h:
            raise RuntimeError("orc_create failed")

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    def set_range(self, lo, hi):
        """Track only bunches [lo, hi) (see orc_set_range)."""
        self.lib.orc_set_range(self.h, int(lo), int(hi))

    def generate_beam(self):
        self.lib.orc_generate_beam(self.h)

    def set_particles(self, ib, soa6):
        a = np.ascontiguousarray(soa6, dtype=np.float64)
        assert a.size == 6 * self.np[ib]
        self.lib.orc_set_particles(self.h, ib, _ptr(a))

    def get_particles(self, ib):
        a = np.empty(6 * self.np[ib])
        self.lib.orc_get_particles(self.h, ib, _ptr(a))
        return a.reshape(6, self.np[ib])

    def prepare(self):
        s = np.zeros(12 * self.nb)
        self.lib.orc_prepare(self.h, _ptr(s))
        return s.reshape(self.nb, 12)

    def deviates_per_turn(self):
        return self.lib.orc_deviates_per_turn(self.h)

    def run(self, nturns, dev_in=None, record=False):
        st = np.zeros(nturns * self.nb * 12)
        dev_out = None
        if record:
            dev_out = np.zeros(max(1, nturns * self.deviates_per_turn()), dtype=np.float32)
        if dev_in is not None:
            dev_in = np.ascontiguousarray(dev_in, dtype=np.float32)
        self.lib.orc_run(self.h, nturns, _ptr(st), _ptr(dev_in), _ptr(dev_out),
                         0 if dev_out is None else dev_out.size)
        st = st.reshape(nturns, self.nb, 12)
        return (st, dev_out) if record else st

    def state(self, ib=0):
        v = np.zeros(2)
        ph = np.zeros(2 * 8)
        self.lib.orc_state(self.h, ib, _ptr(v), _ptr(ph))
        return v, ph

    def trash(self, ib):
        lo, hi = ctypes.c_int(), ctypes.c_int()
        self.lib.orc_trash(self.h, ib, ctypes.byref(lo), ctypes.byref(hi))
        return lo.value, hi.value

    def run_files(self):
        """The rest of the run (NrevTot turns after prepare) with the
        reference's output files written into the work directory
        (refh_run_files); returns the per-turn statistics, invariants, RF
        voltage/phase at each turn's start and the end statistics."""
        L = self.lib
        L.refh_run_files.argtypes = [_vp, _vp, _vp, _vp]
        p = self.params()
        n = int(p.nrev_tot)
        st = np.zeros((n, self.nb, 12))
        ai = np.zeros((n, self.nb, 6))
        vp = np.zeros((n, self.nb, 2))
        end = np.zeros((self.nb, 12))
        rc = L.refh_run_files(_ptr(st), _ptr(ai), _ptr(vp), _ptr(end))
        if rc != 0:
            raise RuntimeError("refh_run_files failed: %d" % rc)
        return st, ai, vp, end

    def output_info(self):
        L = self.lib
        L.refh_output_info.argtypes = [_vp, _vp, _vp, _vp, ctypes.c_int]
        a, b = ctypes.c_long(), ctypes.c_long()
        c = ctypes.c_int()
        out = np.zeros(4096, dtype=np.int32)
        n = L.refh_output_info(ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), _ptr(out), 4096)
        return {"nrev_scan": a.value, "nrev_potentials_out": b.value, "ampinv_out": c.value,
                "bunch_out": out[:n].copy()}

    def ampinv(self, ib):
        out = np.zeros(6)
        self.lib.orc_ampinv.argtypes = [_vp, ctypes.c_int, _vp]
        self.lib.orc_ampinv(self.h, ib, _ptr(out))
        return out

    def enable_beam_ion(self, bi):
        from mbtrack_b200.abi import MbtBeamIon
        self.lib.orc_enable_beam_ion.argtypes = [_vp, _P(MbtBeamIon)]
        self.lib.orc_enable_beam_ion(self.h, ctypes.byref(bi))
        self.bi = bi

    def beam_ion_clouds(self):
        a = np.zeros(self.bi.n_ip * self.nb * 5)
        self.lib.orc_beam_ion_clouds.argtypes = [_vp, _vp]
        self.lib.orc_beam_ion_clouds(self.h, _ptr(a))
        return a.reshape(self.bi.n_ip, self.nb, 5)

    def histograms(self, ib):
        n = self.p.ncell
        arr = [np.zeros(n) for _ in range(6)]
        self.lib.orc_histograms(self.h, ib, *[_ptr(a) for a in arr])
        return arr


def wofz(x, y):
    """Vectorised oracle w(z): returns (re, im, flag)."""
    lib = ctypes.CDLL(build_oracle())
    x = np.ascontiguousarray(x, dtype=np.float64).ravel()
    y = np.ascontiguousarray(y, dtype=np.float64).ravel()
    re, im = np.empty_like(x), np.empty_like(x)
    fl = np.empty(x.size, dtype=np.int32)
    lib.orc_wofz_n.argtypes = [ctypes.c_long, _vp, _vp, _vp, _vp, _vp]
    lib.orc_wofz_n(x.size, _ptr(x), _ptr(y), _ptr(re), _ptr(im), _ptr(fl))
    return re, im, fl


def gauss_field(dx, dy, sx, sy):
    """orc_gauss_field at every point (arrays of equal length)."""
    L = ctypes.CDLL(build_oracle())
    f = L.orc_gauss_field
    f.argtypes = [ctypes.c_double] * 4 + [_P(ctypes.c_double)] * 2
    dx, dy, sx, sy = [np.broadcast_to(np.asarray(a, dtype=np.float64), np.shape(dx)).ravel()
                      for a in (dx, dy, sx, sy)]
    gx, gy = np.zeros(dx.size), np.zeros(dx.size)
    a, b = ctypes.c_double(), ctypes.c_double()
    for i in range(dx.size):
        f(dx[i], dy[i], sx[i], sy[i], ctypes.byref(a), ctypes.byref(b))
        gx[i], gy[i] = a.value, b.value
    return gx, gy


def be_field(dx, dy, sgm_xx_mm, sgm_zz_mm, factdq):
    lib = ctypes.CDLL(build_oracle())
    dx = np.ascontiguousarray(dx, dtype=np.float64).ravel()
    dy = np.ascontiguousarray(dy, dtype=np.float64).ravel()
    ex, ey = np.empty_like(dx), np.empty_like(dx)
    lib.orc_be_field_n.argtypes = [ctypes.c_long, _vp, _vp, ctypes.c_double, ctypes.c_double,
                                   ctypes.c_double, _vp, _vp]
    lib.orc_be_field_n(dx.size, _ptr(dx), _ptr(dy), sgm_xx_mm, sgm_zz_mm, factdq, _ptr(ex), _ptr(ey))
    return ex, ey


class Reference:
    """The reference's own sources run by ref_harness.c."""

    _count = 0

    def __init__(self, conf, fix_rw_beff=True, workdir="/tmp", bunch_range=None, private=True):
        so = build_reference()
        if so is None:
            raise RuntimeError("reference harness unavailable")
        if private:
            # The reference keeps its state in globals and statics (bunch.c's
            # RNG cache among them): load a private copy of the library per
            # instance so instances never share them.
            Reference._count += 1
            priv = os.path.join(tempfile.gettempdir(), "libmbtref_%d_%d.so" % (os.getpid(), Reference._count))
            shutil.copyfile(so, priv)
            self.lib = L = ctypes.CDLL(priv, mode=getattr(os, "RTLD_LOCAL", 0))
            os.unlink(priv)
        else:
            # one instance in this process (a worker of the timed CPU
            # baseline): the built library itself
            self.lib = L = ctypes.CDLL(so, mode=getattr(os, "RTLD_LOCAL", 0))
        L.refh_init.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int]
        L.refh_run.restype = ctypes.c_int
        L.refh_run.argtypes = [ctypes.c_long, _vp, _vp, ctypes.c_long]
        L.refh_prepare.argtypes = [_vp]
        L.refh_get_particles.argtypes = [ctypes.c_int, _vp]
        L.refh_set_particles.argtypes = [ctypes.c_int, _vp]
        L.refh_bunch_info.argtypes = [_vp, _vp, _vp]
        L.refh_state.argtypes = [ctypes.c_int, _vp, _vp]
        L.refh_trash.argtypes = [ctypes.c_int, _vp, _vp]
        L.refh_greens.argtypes = [ctypes.c_int, _vp, _vp, _vp, _vp]
        L.refh_fill_params.argtypes = [_P(MbtParams)]
        L.refh_param_table.argtypes = [_vp, _vp, ctypes.c_int]
        L.refh_set_range.argtypes = [ctypes.c_int, ctypes.c_int]
        if bunch_range is not None:
            L.refh_set_range(int(bunch_range[0]), int(bunch_range[1]))
        self.nb = L.refh_init(conf.encode(), workdir.encode(), int(fix_rw_beff))
        if self.nb <= 0:
            raise RuntimeError("refh_init failed: %d" % self.nb)
        self.bucket = np.zeros(self.nb, dtype=np.int32)
        self.np = np.zeros(self.nb, dtype=np.int32)
        self.ib = np.zeros(self.nb)
        L.refh_bunch_info(_ptr(self.bucket), _ptr(self.np), _ptr(self.ib))
        self.prepared = False

    def deviates_exact(self):
        return bool(self.lib.refh_deviates_exact())

    def get_particles(self, ib):
        a = np.empty(6 * self.np[ib])
        self.lib.refh_get_particles(ib, _ptr(a))
        return a.reshape(6, self.np[ib])

    def set_particles(self, ib, soa6):
        a = np.ascontiguousarray(soa6, dtype=np.float64)
        self.lib.refh_set_particles(ib, _ptr(a))

    def prepare(self):
        s = np.zeros(12 * self.nb)
        self.lib.refh_prepare(_ptr(s))
        self.prepared = True
        return s.reshape(self.nb, 12)

    def params(self):
        p = MbtParams()
        self.lib.refh_fill_params(ctypes.byref(p))
        return p

    def oracle_inputs(self):
        """(params, bucket, np, ib, Gl, Gv, Gh) of this file as the reference's
        own parser and set-up read it: what the C restatement needs."""
        Gl, Gv, Gh, _ = self.greens(0)
        return self.params(), self.bucket.copy(), self.np.copy(), self.ib.copy(), Gl, Gv, Gh

    def greens(self, ib=0):
        p = self.params()
        n = p.ncell
        g = [np.zeros(max(n, 1)) for _ in range(3)]
        planes = np.zeros(3, dtype=np.int32)
        self.lib.refh_greens(ib, _ptr(g[0]), _ptr(g[1]), _ptr(g[2]), _ptr(planes))
        return g[0][:n], g[1][:n], g[2][:n], planes

    def run(self, nturns, record=False, dev_cap=0):
        st = np.zeros(nturns * self.nb * 12)
        dev = np.zeros(max(1, dev_cap), dtype=np.float32) if record else None
        n = self.lib.refh_run(nturns, _ptr(st), _ptr(dev), dev_cap if record else 0)
        st = st.reshape(nturns, self.nb, 12)
        return (st, dev[:n]) if record else st

    def state(self, ib=0):
        v = np.zeros(2)
        ph = np.zeros(16)
        self.lib.refh_state(ib, _ptr(v), _ptr(ph))
        return v, ph

    def trash(self, ib):
        lo, hi = ctypes.c_int(), ctypes.c_int()
        self.lib.refh_trash(ib, ctypes.byref(lo), ctypes.byref(hi))
        return lo.value, hi.value

    def run_files(self):
        """The rest of the run (NrevTot turns after prepare) with the
        reference's output files written into the work directory
        (refh_run_files); returns the per-turn statistics, invariants, RF
        voltage/phase at each turn's start and the end statistics."""
        L = self.lib
        L.refh_run_files.argtypes = [_vp, _vp, _vp, _vp]
        p = self.params()
        n = int(p.nrev_tot)
        st = np.zeros((n, self.nb, 12))
        ai = np.zeros((n, self.nb, 6))
        vp = np.zeros((n, self.nb, 2))
        end = np.zeros((self.nb, 12))
        rc = L.refh_run_files(_ptr(st), _ptr(ai), _ptr(vp), _ptr(end))
        if rc != 0:
            raise RuntimeError("refh_run_files failed: %d" % rc)
        return st, ai, vp, end

    def output_info(self):
        L = self.lib
        L.refh_output_info.argtypes = [_vp, _vp, _vp, _vp, ctypes.c_int]
        a, b = ctypes.c_long(), ctypes.c_long()
        c = ctypes.c_int()
        out = np.zeros(4096, dtype=np.int32)
        n = L.refh_output_info(ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), _ptr(out), 4096)
        return {"nrev_scan": a.value, "nrev_potentials_out": b.value, "ampinv_out": c.value,
                "bunch_out": out[:n].copy()}

    def ampinv(self, ib):
        out = np.zeros(6)
        self.lib.refh_ampinv.argtypes = [ctypes.c_int, _vp]
        self.lib.refh_ampinv(ib, _ptr(out))
        return out


class ReferenceSlices:
    """The reference's slice model (BunchModel = STRONG) with fast beam-ion
    interaction, run by ref_ws_harness.c.  fix_ibunch sets the bunch
    currents the reference's slice-model manager leaves at zero."""

    def __init__(self, conf, fix_ibunch=True, workdir="/tmp"):
        so = build_reference()
        if so is None:
            raise RuntimeError("reference harness unavailable")
        Reference._count += 1
        priv = os.path.join(tempfile.gettempdir(), "libmbtref_%d_%d.so" % (os.getpid(), Reference._count))
        shutil.copyfile(so, priv)
        self.lib = L = ctypes.CDLL(priv, mode=getattr(os, "RTLD_LOCAL", 0))
        os.unlink(priv)
        L.refws_init.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int]
        L.refws_info.argtypes = [_vp] * 6
        L.refws_particles.argtypes = [_vp]
        L.refws_get_slices.argtypes = [_vp]
        L.refws_set_slices.argtypes = [_vp]
        L.refws_run.argtypes = [ctypes.c_long, _vp, _vp, _vp, _vp]
        L.refws_bunch_fields.argtypes = [ctypes.c_int, _vp, _vp]
        L.refws_interp.argtypes = [ctypes.c_int, ctypes.c_int, _vp, _vp, ctypes.c_int, _vp]
        self.nb = L.refws_init(conf.encode(), workdir.encode(), int(fix_ibunch))
        if self.nb <= 0:
            raise RuntimeError("refws_init failed: %d" % self.nb)
        oi = np.zeros(9, np.int32)
        od = np.zeros(11)
        L.refws_info(_ptr(oi), _ptr(od), None, None, None, None)
        self.nslc, self.slices, self.ngrid, self.offst, self.np, self.nharm, self.nmultit, self.fbii, self.rw = \
            [int(v) for v in oi]
        (self.agLOCx, self.agLOCz, self.agABSx, self.agABSz, self.deltT, self.factBE, self.factF, self.Ldmsgm,
         self.sgm_xx, self.sgm_zz, self.sgmatau) = [float(v) for v in od]
        S, G = self.slices, self.ngrid
        self.bucket = np.zeros(self.nb, np.int32)
        self.ibunch = np.zeros(self.nb)
        self.npop = np.zeros(S, np.int32)
        self.nofe = np.zeros((S, G, G), np.int32)
        L.refws_info(_ptr(oi), _ptr(od), _ptr(self.bucket), _ptr(self.ibunch), _ptr(self.npop), _ptr(self.nofe))
        self.nmon_done = 0

    def params(self):
        """mbt_ws_params from the reference's set-up: base through
        refh_fill_params (the same globals), the slice-model values from
        refws_info."""
        w = MbtWsParams()
        self.lib.refh_fill_params.argtypes = [_P(MbtParams)]
        self.lib.refh_fill_params(ctypes.byref(w.base))
        w.nslc, w.fbii, w.np, w.ngrid, w.ndivs = self.nslc, self.fbii, self.np, self.ngrid, 3
        w.sgm_xx, w.sgm_zz, w.sgmatau, w.max_tau, w.dtau = self.sgm_xx, self.sgm_zz, self.sgmatau, 7.0, 0.3
        w.agLOCx, w.agLOCz, w.agABSx, w.agABSz = self.agLOCx, self.agLOCz, self.agABSx, self.agABSz
        w.deltT, w.factBE, w.factF, w.Ldmsgm = self.deltT, self.factBE, self.factF, self.Ldmsgm
        w.Gamma = 1957.0 * w.base.E0
        w.kick_factor = 1e2
        return w

    def particles(self):
        a = np.zeros((6, self.np))
        self.lib.refws_particles(_ptr(a))
        return a

    def files(self, on=True):
        """The manager's writers into the work directory (refws_files)."""
        self.lib.refws_files(int(on))

    def finish(self):
        self.lib.refws_finish()

    def write_distribution(self):
        if self.lib.refws_write_distribution() != 0:
            raise RuntimeError("refws_write_distribution failed")

    def slices_state(self):
        a = np.zeros((self.nb, 6, self.slices))
        self.lib.refws_get_slices(_ptr(a))
        return a

    def set_slices(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        self.lib.refws_set_slices(_ptr(a))

    def run(self, nturns, nrev_mon, rev0=0):
        """Per-turn outputs of refws_run: cm (n, nb, 6), ion (n, nb, 2),
        zcm (n, nharm), stats (monitor turns, nb, 18)."""
        nmon = sum(1 for r in range(rev0, rev0 + nturns) if r % nrev_mon == 0)
        cm = np.zeros((nturns, self.nb, 6))
        ion = np.zeros((nturns, self.nb, 2))
        zcm = np.zeros((nturns, self.nharm))
        st = np.zeros((max(nmon, 1), self.nb, 18))
        rc = self.lib.refws_run(nturns, _ptr(cm), _ptr(ion), _ptr(zcm), _ptr(st))
        if rc != 0:
            raise RuntimeError("refws_run failed: %d" % rc)
        return cm, ion, zcm, st[:nmon]

    def bunch_fields(self, ib):
        n = self.slices * self.ngrid * self.ngrid
        e = np.zeros((n, 2))
        ions = np.zeros((5, n))
        self.lib.refws_bunch_fields(ib, _ptr(e), _ptr(ions))
        return e, ions

    def interp(self, ib, icell, x, y):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.ascontiguousarray(y, dtype=np.float64)
        out = np.zeros((x.size, 2))
        self.lib.refws_interp(ib, icell, _ptr(x), _ptr(y), x.size, _ptr(out))
        return out


class OracleSlices:
    """The C restatement of the slice model (ws_oracle.c)."""

    def __init__(self, w, bucket, ibunch, npop, nofe):
        self.lib = L = ctypes.CDLL(build_oracle())
        L.ows_create.restype = _vp
        L.ows_create.argtypes = [_P(MbtWsParams), ctypes.c_int, _vp, _vp, _vp, _vp]
        L.ows_destroy.argtypes = [_vp]
        L.ows_set_slices.argtypes = [_vp, _vp]
        L.ows_get_slices.argtypes = [_vp, _vp]
        L.ows_run.argtypes = [_vp, ctypes.c_long, _vp, _vp, _vp, _vp]
        L.ows_bunch_fields.argtypes = [_vp, ctypes.c_int, _vp, _vp]
        L.ows_interp_n.argtypes = [_vp, ctypes.c_int, ctypes.c_int, _vp, _vp, ctypes.c_int, _vp]
        self.w = w
        self.nb = len(bucket)
        self.S = w.slices
        self.nion = self.S * w.ngrid * w.ngrid
        self.nharm = w.base.nharm
        self.rev = 0
        self._keep = [np.ascontiguousarray(bucket, dtype=np.int32), np.ascontiguousarray(ibunch, dtype=np.float64),
                      np.ascontiguousarray(npop, dtype=np.int32), np.ascontiguousarray(nofe, dtype=np.int32)]
        self.o = L.ows_create(ctypes.byref(w), self.nb, *[_ptr(a) for a in self._keep])
        if not self.o:
            raise RuntimeError("ows_create failed")

    def __del__(self):
        if getattr(self, "o", None):
            self.lib.ows_destroy(self.o)
            self.o = None

    def set_slices(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        self.lib.ows_set_slices(self.o, _ptr(a))

    def slices_state(self):
        a = np.zeros((self.nb, 6, self.S))
        self.lib.ows_get_slices(self.o, _ptr(a))
        return a

    def run(self, nturns):
        nmon = sum(1 for r in range(self.rev, self.rev + nturns) if r % self.w.base.nrev_mon == 0)
        cm = np.zeros((nturns, self.nb, 6))
        ion = np.zeros((nturns, self.nb, 2))
        zcm = np.zeros((nturns, self.nharm))
        st = np.zeros((max(nmon, 1), self.nb, 18))
        rc = self.lib.ows_run(self.o, nturns, _ptr(cm), _ptr(ion), _ptr(zcm), _ptr(st))
        if rc != 0:
            raise RuntimeError("ows_run failed: %d" % rc)
        self.rev += nturns
        return cm, ion, zcm, st[:nmon]

    def bunch_fields(self, ib):
        e = np.zeros((self.nion, 2))
        ions = np.zeros((5, self.nion))
        self.lib.ows_bunch_fields(self.o, ib, _ptr(e), _ptr(ions))
        return e, ions

    def interp(self, ib, icell, x, y):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.ascontiguousarray(y, dtype=np.float64)
        out = np.zeros((x.size, 2))
        self.lib.ows_interp_n(self.o, ib, icell, _ptr(x), _ptr(y), x.size, _ptr(out))
        return out


def slice_beam(w, soa6):
    """ows_slice_beam: (npop[S], nofe[S, G, G], cm4[4, S]) of soa6."""
    L = ctypes.CDLL(build_oracle())
    L.ows_slice_beam.argtypes = [_P(MbtWsParams), _vp, ctypes.c_int, _vp, _vp, _vp]
    soa6 = np.ascontiguousarray(soa6, dtype=np.float64)
    S, G = w.slices, w.ngrid
    npop = np.zeros(S, np.int32)
    nofe = np.zeros((S, G, G), np.int32)
    cm4 = np.zeros((4, S))
    if L.ows_slice_beam(ctypes.byref(w), _ptr(soa6), soa6.shape[1], _ptr(npop), _ptr(nofe), _ptr(cm4)) != 0:
        raise RuntimeError("ows_slice_beam failed")
    return npop, nofe, cm4


def mlp_forward(params, abr):
    """orc_mlp_forward: the network's outputs for inputs abr (n x 3)."""
    L = ctypes.CDLL(build_oracle())
    p = np.ascontiguousarray(params, dtype=np.float32)
    x = np.ascontiguousarray(abr, dtype=np.float32)
    out = np.zeros((len(x), 2), dtype=np.float32)
    L.orc_mlp_forward.argtypes = [_vp, ctypes.c_long, _vp, _vp]
    L.orc_mlp_forward(_ptr(p), len(x), _ptr(x), _ptr(out))
    return out


def mlp_gradient(params, abr, tgt):
    """orc_mlp_gradient: (gradient, loss) of one batch."""
    L = ctypes.CDLL(build_oracle())
    p = np.ascontiguousarray(params, dtype=np.float32)
    x = np.ascontiguousarray(abr, dtype=np.float32)
    t = np.ascontiguousarray(tgt, dtype=np.float32)
    g = np.zeros(p.size, dtype=np.float32)
    L.orc_mlp_gradient.argtypes = [_vp, ctypes.c_int, _vp, _vp, _vp]
    L.orc_mlp_gradient.restype = ctypes.c_double
    loss = L.orc_mlp_gradient(_ptr(p), len(x), _ptr(x), _ptr(t), _ptr(g))
    return g, loss
