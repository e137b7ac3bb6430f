"""ctypes mirror of the C-ABI structures declared in include/mbt.h.

The layouts must match the C declarations field for field; libmbt exports
``mbt_params_size()`` so the loader can check the size at import time.
"""
import ctypes

MBT_MAX_RES = 32
MBT_MAX_LR = 8
MBT_MAX_AHC = 8
MBT_MAX_NCELL = 1024

MBT_OK = 0
MBT_ERR_INVALID = -1
MBT_ERR_CUDA = -2
MBT_ERR_NOMEM = -3
MBT_ERR_CONFIG = -4
MBT_ERR_STATE = -5
MBT_ERR_TIMEOUT = -6
MBT_ERR_NODEVICE = -7

MBT_NOISE_PHILOX = 0
MBT_NOISE_INJECTED = 1

LON, HOR, VER = 0, 1, 2

_d = ctypes.c_double
_i = ctypes.c_int
_l = ctypes.c_long


class MbtParams(ctypes.Structure):
    """mbt_params (include/mbt.h)."""
    _fields_ = [
        ("nharm", _i), ("E0", _d), ("T0", _d), ("wrf", _d), ("Vrf0", _d),
        ("phai0", _d), ("Urad", _d), ("De", _d), ("ac", _d),
        ("QH0", _d), ("QV0", _d), ("Gzix", _d), ("Gziz", _d),
        ("CHH", _d), ("CHV", _d), ("CVH", _d), ("CVV", _d),
        ("amp_dep_qv", _i),
        ("beta1", _d * 3), ("alpha1", _d * 3), ("gamma1", _d * 3),
        ("dispH1", _d), ("disppH1", _d),
        ("taue", _d), ("taux", _d), ("tauz", _d),
        ("Lc", _d), ("rhorw", _d),
        ("beffH", _d * 2), ("beffV", _d * 2), ("beffL", _d * 2),
        ("Iring", _d),
        ("ideal_hc", _i), ("m_aHC", _i), ("phi_n", _d), ("HC_k", _d),
        ("n_active_hc", _i),
        ("ahc_vpeak", _d * MBT_MAX_AHC), ("ahc_nhc", _d * MBT_MAX_AHC),
        ("ahc_phi", _d * MBT_MAX_AHC),
        ("track_plane", _i * 3), ("quantum", _i), ("rw_long", _i),
        ("Nmlt", _i), ("triggerRW", _i), ("nrev_tot", _l), ("nrev_mon", _l),
        ("scan", _i), ("nscan", _l), ("nrev_scan", _l),
        ("scan_start", _d), ("scan_step", _d),
        ("np_model", _i), ("iseed", _i * 3),
        ("pos_offset", _d * 3), ("slope_offset", _d * 3),
        ("pos_sgm", _d * 3), ("slope_sgm", _d * 3), ("correlate", _d * 3),
        ("ncell", _i), ("nsigma", _d), ("dT", _d), ("sigma_tau", _d),
        ("RsisL", _d), ("aindL", _d),
        ("planeL", _i), ("planeV", _i), ("planeH", _i),
        ("n_lr", _i * 3),
        ("lr_Rs", (_d * MBT_MAX_LR) * 3), ("lr_wr", (_d * MBT_MAX_LR) * 3),
        ("lr_Q", (_d * MBT_MAX_LR) * 3),
        ("lr_init_turns", _i),
        ("rffb", _i), ("rffb_resonator", _i), ("rffb_len", _i),
        ("rffb_off_after_init", _i),
        ("rffb_vrf_design", _d), ("rffb_phi0_design", _d), ("rffb_gain", _d), ("rffb_delay", _i),
    ]

    def copy(self):
        c = MbtParams()
        ctypes.memmove(ctypes.byref(c), ctypes.byref(self), ctypes.sizeof(self))
        return c


class MbtState(ctypes.Structure):
    """mbt_state (include/mbt.h)."""
    _fields_ = [
        ("turn", _l), ("Vrf0", _d), ("phai0", _d),
        ("phasor", ((_d * 2) * MBT_MAX_LR) * 3),
        ("n_trash_low", _i), ("n_trash_high", _i),
    ]


class MbtOutputCfg(ctypes.Structure):
    """mbt_output_cfg (include/mbt.h)."""
    _fields_ = [
        ("jobtitle", ctypes.c_char * 80),
        ("gendst_file", (ctypes.c_char * 1024) * 3),
        ("nrev_potentials_out", _l), ("ampinv_out", _i), ("n_out", _i),
    ]


MBT_WRITER_OWN_AMPINV = 1


class MbtBeamIon(ctypes.Structure):
    """mbt_beam_ion (include/mbt.h)."""
    _fields_ = [
        ("n_ip", _i), ("ions_per_passage", _i), ("gas_A", _d), ("pressure", _d),
        ("sigma_ion", _d), ("seed", ctypes.c_uint64), ("surrogate", _i), ("audit_fraction", _d),
    ]


class MbtWsParams(ctypes.Structure):
    """mbt_ws_params (include/mbt_ws.h)."""
    _fields_ = [
        ("base", MbtParams),
        ("nslc", _i), ("fbii", _i), ("np", _i), ("ngrid", _i), ("ndivs", _i),
        ("sgm_xx", _d), ("sgm_zz", _d), ("sgmatau", _d), ("max_tau", _d), ("dtau", _d),
        ("agLOCx", _d), ("agLOCz", _d), ("agABSx", _d), ("agABSz", _d),
        ("deltT", _d), ("factBE", _d), ("factF", _d), ("Ldmsgm", _d), ("Gamma", _d),
        ("sgm_in", _d * 6), ("cm_in", _d * 6), ("kick_factor", _d),
    ]

    @property
    def slices(self):
        return 2 * self.nslc + 1


def params_to_dict(p):
    """Flatten an MbtParams into {field: scalar or nested list}."""
    out = {}
    for name, _ in MbtParams._fields_:
        v = getattr(p, name)
        if isinstance(v, ctypes.Array):
            v = [list(x) if isinstance(x, ctypes.Array) else x for x in v]
        out[name] = v
    return out


def params_from_dict(d):
    p = MbtParams()
    for name, _ in MbtParams._fields_:
        if name not in d:
            continue
        v = d[name]
        cur = getattr(p, name)
        if isinstance(cur, ctypes.Array):
            for i, x in enumerate(v):
                if isinstance(cur[i], ctypes.Array):
                    for j, y in enumerate(x):
                        cur[i][j] = y
                else:
                    cur[i] = x
        else:
            setattr(p, name, v)
    return p
