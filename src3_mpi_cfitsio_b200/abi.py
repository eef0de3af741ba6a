"""ctypes mirror of include/mcrt_b200.h.

The structs here are byte-for-byte the C structs of the engine's C ABI (the
boundary a Fortran ``iso_c_binding`` interface binds).
``Bundle`` keeps the numpy arrays alive for as long as a struct points at
them.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

MCRT_OK = 0
MCRT_NDG2 = 10
MCRT_NO = 8
MCRT_NSCALARS = 8
MCRT_NCOUNTERS = 16
PREC_FP64 = 0
PREC_MIXED = 1

SCALARS = ["flux", "sflux", "nscat", "tot", "scount", "dscount", "aflux", "abflux"]
COUNTERS = ["packets", "crossings", "interactions", "scatters", "peels", "peel_cross",
            "peel_binned", "geom_fail", "resets", "killed", "exited", "starhits",
            "peel_resets", "peel_jobs", "waves", "launches"]

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_fp = C.POINTER(C.c_float)
_lp = C.POINTER(C.c_int64)


class Config(C.Structure):
    _fields_ = [(n, C.c_int32) for n in (
        "nrg", "ntg", "npg", "nopac", "nlammax", "nT", "nnu", "nhnu",
        "nfreq", "nmu", "nph", "nap", "npeel", "nxhst",
        "output_imcube", "partial_peeloff", "limb", "iplanckst", "idust", "ilucy",
        "iffuv", "ispot", "nspot", "pad0")] + [(n, C.c_double) for n in (
        "rstar", "tstar", "tstarave", "tshock", "fspot", "accfrac", "accfrac2",
        "isrf_frac", "rddust", "rmaxi", "numin", "lnurat", "autors", "ifuv_ori",
        "cspot1", "sspot1", "scspot1", "ssspot1", "cspot2", "sspot2", "scspot2",
        "ssspot2", "csprad")] + [(n, C.c_int32) for n in ("output_imfilt", "nfilt", "nwfiltmax", "pad_filt",
                                                           "output_imsparse", "sparse_dim", "sparse_nlev",
                                                           "sparse_nnu")] + [
        (n, C.c_float) for n in ("sparse_lognu_min", "sparse_lognu_max")]


GRID_FIELDS = [("rarr", _dp), ("r2arr", _dp), ("thetarr", _dp), ("costarr", _dp),
               ("sintarr", _dp), ("tan2arr", _dp), ("phiarr", _dp), ("aarr", _dp),
               ("barr", _dp), ("densarr", _dp), ("findopac", _ip), ("diffus", _ip),
               ("diffdir", _ip), ("tdust", _dp), ("vcell", _dp), ("ravearr", _dp),
               ("Ldint", _dp), ("hdisk", _dp), ("vrarr", _dp), ("vthetarr", _dp), ("divvarr", _dp),
               ("imean", _ip)]


class Grid(C.Structure):
    _fields_ = GRID_FIELDS


TABLE_FIELDS = [("nlambda", _ip), ("nudust", _dp), ("kappad", _dp), ("adust", _dp),
                ("gdust", _dp), ("pldust", _dp), ("kappav", _dp), ("kapint", _dp),
                ("lTint", _dp), ("Tint", _dp), ("nuint", _dp), ("kappap", _dp),
                ("kappar", _dp), ("atmosnu", _dp), ("hnuint", _dp), ("lognu", _dp),
                ("loghnu", _dp), ("aperture2", _dp), ("u", _dp), ("coste_arr", _dp),
                ("sinte_arr", _dp), ("cospe_arr", _dp), ("sinpe_arr", _dp),
                ("limb_prob", _dp), ("mueller", _dp), ("narr", C.c_int32), ("pad_mueller", C.c_int32),
                ("isrf", _dp), ("nisrf", C.c_int32), ("pad_isrf", C.c_int32),
                ("draine", _dp), ("nemit", C.c_int32), ("ndraine", C.c_int32),
                ("nwfilt", _ip), ("filtwave", _dp), ("filtphi", _dp), ("sparse_levels", _fp)]


class Tables(C.Structure):
    _fields_ = TABLE_FIELDS


CELL_I = ["nabs", "dbig", "dsg", "killed"]
CELL_D = ["dtauabs", "fuvmean"]
SED = ["si", "sq", "su", "sv", "si2", "sq2", "su2", "sv2", "nums", "aveinc"]
PSED = ["ti", "tq", "tu", "tv", "ti2", "tq2", "tu2", "tv2", "numt"]
IMG = ["image_m_i", "image_m_q", "image_m_u", "image_m_v"]
IMGB = ["image_b_i", "image_b_q", "image_b_u", "image_b_v", "image_b_d", "image_b_s", "image_b_e", "image_b_o"]
IMGS = ["image_ms_i", "image_ms_q", "image_ms_u", "image_ms_v"]


class Tallies(C.Structure):
    _fields_ = ([(n, _ip) for n in CELL_I] + [(n, _dp) for n in CELL_D] +
                [(n, _fp) for n in SED] + [(n, _fp) for n in PSED] +
                [(n, _fp) for n in IMG] + [("scalars", _dp), ("counters", _lp)] +
                [(n, _fp) for n in IMGB] + [(n, _fp) for n in IMGS])


class PacketLog(C.Structure):
    _fields_ = [("iphot", C.c_int64)] + [(n, C.c_int32) for n in (
        "nscat", "nabs", "ncross", "nstar", "status", "ir", "it", "ip", "ndraws",
        "iflag", "i_orig", "pad")] + [(n, C.c_double) for n in (
        "nub", "cost", "phi", "sip", "sqp", "sup", "svp", "xp", "yp", "zp")]


class DensityParams(C.Structure):
    """mcrt_density_params (parameters of mcrt_model_density)."""
    _fields_ = [(n, C.c_double) for n in (
        "rstar", "autors", "rddust", "rmax", "rmaxd", "massd", "a_exp", "b_exp", "h100_au", "rate", "rc",
        "massc", "rhoamb", "thet1_deg", "ex1", "rhoconst1")]


class DeviceTallies(C.Structure):
    """mcrt_device_tallies: device addresses of the three tally segments."""
    _fields_ = [("f64", C.c_void_p), ("n_f64", C.c_int64), ("u64", C.c_void_p), ("n_u64", C.c_int64),
                ("i32", C.c_void_p), ("n_i32", C.c_int64)]


def _ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


class Bundle:
    """Config/Grid/Tables structs over a Model's arrays (kept alive here)."""

    def __init__(self, model):
        self.model = model
        cfg = Config()
        for name, _ in Config._fields_:
            if name == "pad0":
                continue
            v = model.config.get(name, 0)
            setattr(cfg, name, v)
        self.config = cfg
        self._keep = []
        self.grid = self._struct(Grid, model.grid)
        self.tables = self._struct(Tables, model.tables)

    def _struct(self, cls, arrays):
        s = cls()
        for name, ptype in cls._fields_:
            a = arrays.get(name)
            if a is None:
                continue
            if ptype is C.c_int32:          # scalar member
                setattr(s, name, int(a))
                continue
            if ptype is C.c_float:          # scalar member
                setattr(s, name, float(a))
                continue
            if ptype is _ip:
                a = np.ascontiguousarray(a, dtype=np.int32)
                ct = C.c_int32
            elif ptype is _fp:
                a = np.ascontiguousarray(a, dtype=np.float32)
                ct = C.c_float
            else:
                a = np.ascontiguousarray(a, dtype=np.float64)
                ct = C.c_double
            self._keep.append(a)
            setattr(s, name, _ptr(a, ct))
        return s


class TallyArrays:
    """Caller-owned host arrays for one tally download."""

    def __init__(self, cfg: Config, images: bool = True):
        ncell = cfg.nrg * cfg.ntg * cfg.npg
        nsed = cfg.nfreq * cfg.nmu * cfg.nph * cfg.nap * MCRT_NO
        npsed = cfg.nfreq * cfg.npeel * cfg.nap * MCRT_NO
        nimg = cfg.npeel * cfg.nxhst * cfg.nxhst * cfg.nfreq
        self.cfg = cfg
        self.arrays: dict[str, np.ndarray] = {}
        for n in CELL_I:
            self.arrays[n] = np.zeros(ncell, np.int32)
        for n in CELL_D:
            self.arrays[n] = np.zeros(ncell, np.float64)
        for n in SED:
            self.arrays[n] = np.zeros(nsed, np.float32)
        for n in PSED:
            self.arrays[n] = np.zeros(npsed, np.float32)
        if images and cfg.output_imcube:
            for n in IMG:
                self.arrays[n] = np.zeros(nimg, np.float32)
        if images and cfg.output_imfilt:
            nimgb = cfg.npeel * cfg.nxhst * cfg.nxhst * cfg.nfilt
            for n in IMGB:
                self.arrays[n] = np.zeros(nimgb, np.float32)
        if images and cfg.output_imsparse:
            nims = cfg.sparse_dim * cfg.sparse_dim * cfg.sparse_nnu * cfg.sparse_nlev * cfg.npeel
            for n in IMGS:
                self.arrays[n] = np.zeros(nims, np.float32)
        self.arrays["scalars"] = np.zeros(MCRT_NSCALARS, np.float64)
        self.arrays["counters"] = np.zeros(MCRT_NCOUNTERS, np.int64)
        t = Tallies()
        for name, ptype in Tallies._fields_:
            a = self.arrays.get(name)
            if a is not None:
                setattr(t, name, a.ctypes.data_as(ptype))
        self.struct = t

    def __getitem__(self, k):
        return self.arrays[k]

    def add_(self, other: "TallyArrays"):
        """Sum another tally set into this one in place (the struct keeps
        pointing at the same arrays): integers and FP64 exactly, the REAL
        arrays in FP64 with one rounding."""
        for k, a in self.arrays.items():
            b = other.arrays[k]
            if a.dtype == np.float32:
                a[:] = (a.astype(np.float64) + b).astype(np.float32)
            else:
                a += b
        return self

    def scalars(self) -> dict:
        return dict(zip(SCALARS, self.arrays["scalars"].tolist()))

    def counters(self) -> dict:
        return dict(zip(COUNTERS, self.arrays["counters"].tolist()))

    def shaped(self, name):
        c = self.cfg
        a = self.arrays[name]
        if name in CELL_I or name in CELL_D:
            return a.reshape((c.nrg, c.ntg, c.npg), order="F")
        if name in SED:
            return a.reshape((c.nfreq, c.nmu, c.nph, c.nap, MCRT_NO), order="F")
        if name in PSED:
            return a.reshape((c.nfreq, c.npeel, c.nap, MCRT_NO), order="F")
        if name in IMG:
            return a.reshape((c.npeel, c.nxhst, c.nxhst, c.nfreq), order="F")
        if name in IMGB:
            return a.reshape((c.npeel, c.nxhst, c.nxhst, c.nfilt), order="F")
        if name in IMGS:
            return a.reshape((c.sparse_dim, c.sparse_dim, c.sparse_nnu, c.sparse_nlev, c.npeel), order="F")
        return a


def packet_log_array(n: int):
    return (PacketLog * n)()


def packet_log_to_numpy(log) -> dict:
    out = {}
    for name, _ in PacketLog._fields_:
        out[name] = np.array([getattr(r, name) for r in log])
    return out
