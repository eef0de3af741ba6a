"""Python handle on the CPU oracle (TEST INFRASTRUCTURE ONLY).

Loads oracle/_build/libmcrt_oracle.so (built by oracle/Makefile) and runs the
FP64 restatement of the reference's packet loop on host threads.  Only the
tests, ``__graft_entry__.smoke`` and the CPU-baseline leg of bench.py use it,
always as the checker or the baseline, never as the engine.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from src3_mpi_cfitsio_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libmcrt_oracle.so")
_lib = None
_native = False


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def native_lib() -> str:
    """The oracle built with -march=native for THIS host (timing only; the
    arithmetic is the same: FMA contraction stays off).  The file name
    carries a hash of the host's CPU model and flags, so a copy built on
    another machine is never loaded here."""
    import hashlib
    flags = ""
    try:
        with open("/proc/cpuinfo") as f:
            flags = next((ln for ln in f if ln.startswith("flags")), "")
    except OSError:
        pass
    tag = hashlib.sha1((cpu_model() + flags).encode()).hexdigest()[:12]
    out = os.path.join(HERE, "_build", f"libmcrt_oracle_native_{tag}.so")
    if not os.path.exists(out):
        subprocess.run(["make", "-s", "-C", HERE, "native", f"NATIVE_OUT={out}"], check=True)
    return out


def use_native() -> None:
    """Switch this module to the host-native build (bench.py's CPU legs)."""
    global _lib, _native
    if not _native:
        _lib = None
        _native = True


def load():
    global _lib
    if _lib is None:
        if not _native and not os.path.exists(LIB):
            build()
        lib = C.CDLL(native_lib() if _native else LIB)
        lib.oracle_run.argtypes = [C.POINTER(abi.Config), C.POINTER(abi.Grid), C.POINTER(abi.Tables),
                                   C.c_int64, C.c_int64, C.c_int64, C.c_int32, C.c_int32,
                                   C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                   C.POINTER(abi.Tallies), C.POINTER(abi.PacketLog), C.c_int64,
                                   C.POINTER(C.c_double)]
        lib.oracle_run.restype = C.c_int
        D = C.POINTER(C.c_double)
        lib.oracle_adjoint.argtypes = [C.POINTER(abi.Config), C.POINTER(abi.Grid), C.POINTER(abi.Tables),
                                       C.c_int64, C.c_int64, C.c_int64, C.c_int32, C.c_int32, C.c_int32,
                                       C.c_int32, C.c_int32, D, D, D, D]
        lib.oracle_adjoint.restype = C.c_int
        lib.oracle_adjoint_cv.argtypes = lib.oracle_adjoint.argtypes + [D, C.c_int32, D, D]
        lib.oracle_adjoint_cv.restype = C.c_int
        lib.oracle_rep_draine.argtypes = [C.POINTER(abi.Tables), C.c_int32, C.c_int64, C.c_int32, C.c_int32, D]
        lib.oracle_rep_draine.restype = C.c_int
        lib.oracle_rng.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_int64, C.c_int32,
                                   C.POINTER(C.c_double), C.POINTER(C.c_int32)]
        lib.oracle_inczeta.argtypes = [C.POINTER(C.c_double)]
        lib.oracle_tfinal.argtypes = [C.POINTER(abi.Config), C.POINTER(abi.Grid), C.POINTER(abi.Tables),
                                      C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int32, C.c_int32,
                                      C.POINTER(C.c_double), C.POINTER(C.c_int32), C.POINTER(C.c_double)]
        lib.oracle_tfinal.restype = C.c_int
        lib.oracle_setdiffus.argtypes = [C.POINTER(abi.Config), C.POINTER(abi.Grid), C.POINTER(abi.Tables),
                                         C.c_int32, C.c_double, C.c_double, C.POINTER(C.c_double),
                                         C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_double)]
        lib.oracle_setdiffus.restype = C.c_int
        D = C.POINTER(C.c_double)
        lib.oracle_setemiss.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_int32), D, D, D, C.c_int32,
                                        C.c_int32, D, D, D, D, D, D, C.POINTER(C.c_int64), C.c_int32]
        lib.oracle_setemiss.restype = C.c_int
        _lib = lib
    return _lib


def run(bundle: abi.Bundle, np_total: int, lo: int = 1, hi: int | None = None, *, ipeel: int = 1,
        iteration: int = 1, seeds=(12345678, 87654321), generator: int = 1,
        threads: int | None = None, nlog: int = 0, images: bool = True):
    """Run packets lo..hi of an np_total-packet iteration; returns (tallies, log)."""
    lib = load()
    hi = np_total if hi is None else hi
    threads = threads or os.cpu_count() or 1
    tal = abi.TallyArrays(bundle.config, images=images)
    log = abi.packet_log_array(nlog) if nlog > 0 else None
    c = bundle.config
    tal.tdust = np.zeros(c.nrg * c.ntg * c.npg, np.float64)
    rc = lib.oracle_run(C.byref(bundle.config), C.byref(bundle.grid), C.byref(bundle.tables),
                        np_total, lo, hi, iteration, ipeel, seeds[0], seeds[1], generator, threads,
                        C.byref(tal.struct), log, nlog, tal.tdust.ctypes.data_as(C.POINTER(C.c_double)))
    if rc != 0:
        raise RuntimeError(f"oracle_run failed with code {rc}")
    return tal, log


def rng(seed1: int, seed2: int, generator: int, block: int, n: int):
    lib = load()
    out = np.zeros(n, np.float64)
    seeds = np.zeros(2, np.int32)
    lib.oracle_rng(seed1, seed2, generator, block, n, out.ctypes.data_as(C.POINTER(C.c_double)),
                   seeds.ctypes.data_as(C.POINTER(C.c_int32)))
    return out, seeds


def inczeta():
    out = np.zeros(145, np.float64)
    load().oracle_inczeta(out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


def tfinal(bundle: abi.Bundle, dtauabs: np.ndarray, nphot: int, iteration: int, tdave: np.ndarray,
           tdust_now: np.ndarray | None = None):
    lib = load()
    td = np.ascontiguousarray(tdave, dtype=np.float64).copy()
    da = np.ascontiguousarray(dtauabs, dtype=np.float64)
    tn = None if tdust_now is None else np.ascontiguousarray(tdust_now, dtype=np.float64)
    conv = C.c_int32(0)
    sig = np.zeros(3, np.float64)
    rc = lib.oracle_tfinal(C.byref(bundle.config), C.byref(bundle.grid), C.byref(bundle.tables),
                           da.ctypes.data_as(C.POINTER(C.c_double)),
                           None if tn is None else tn.ctypes.data_as(C.POINTER(C.c_double)), nphot, iteration,
                           td.ctypes.data_as(C.POINTER(C.c_double)), C.byref(conv),
                           sig.ctypes.data_as(C.POINTER(C.c_double)))
    if rc != 0:
        raise RuntimeError(f"oracle_tfinal failed with code {rc}")
    return td, sig


def setdiffus(bundle: abi.Bundle, iteration: int, massd: float, rmaxd: float, tdave: np.ndarray):
    """setdiffus (setdiffus_5.f90:1-132) and gridset's tdust reset
    (gridset_5_model13new.f90:1855-1866): returns (diffus, diffdir, tdust),
    Fortran-order flat arrays."""
    lib = load()
    td = np.ascontiguousarray(tdave, dtype=np.float64)
    n = td.size
    dif = np.zeros(n, np.int32)
    ddir = np.zeros(n, np.int32)
    tdust = np.zeros(n, np.float64)
    I = C.POINTER(C.c_int32)
    rc = lib.oracle_setdiffus(C.byref(bundle.config), C.byref(bundle.grid), C.byref(bundle.tables), iteration,
                              float(massd), float(rmaxd), td.ctypes.data_as(C.POINTER(C.c_double)),
                              dif.ctypes.data_as(I), ddir.ctypes.data_as(I), tdust.ctypes.data_as(C.POINTER(C.c_double)))
    if rc != 0:
        raise RuntimeError(f"oracle_setdiffus failed with code {rc}")
    return dif, ddir, tdust


def adjoint(bundle: abi.Bundle, np_total: int, lam_psed: np.ndarray, lam_img: np.ndarray | None = None,
            lo: int = 1, hi: int | None = None, *, iteration: int = 1, seeds=(12345678, 87654321),
            generator: int = 1, threads: int | None = None):
    """Path-replay adjoint of L = sum lam_psed*ti + sum lam_img*image_m_i:
    returns (grad [ncell*10] = dL/dlog(rho) per cell and component id,
    Fortran order, and L).  Diffusion surfaces keep their start-of-iteration
    temperature (no within-iteration heating)."""
    lib = load()
    hi = np_total if hi is None else hi
    threads = threads or os.cpu_count() or 1
    c = bundle.config
    ncell = c.nrg * c.ntg * c.npg
    lp = np.ascontiguousarray(lam_psed, dtype=np.float64)
    li = None if lam_img is None else np.ascontiguousarray(lam_img, dtype=np.float64)
    grad = np.zeros(ncell * 10, np.float64)
    obj = C.c_double(0.0)
    D = C.POINTER(C.c_double)
    rc = lib.oracle_adjoint(C.byref(bundle.config), C.byref(bundle.grid), C.byref(bundle.tables), np_total, lo, hi,
                            iteration, seeds[0], seeds[1], generator, threads, lp.ctypes.data_as(D),
                            li.ctypes.data_as(D) if li is not None else None, grad.ctypes.data_as(D), C.byref(obj))
    if rc != 0:
        raise RuntimeError(f"oracle_adjoint failed with code {rc}")
    return grad, obj.value


def adjoint_cv(bundle: abi.Bundle, np_total: int, lam_psed: np.ndarray, lam_img: np.ndarray | None = None,
               lo: int = 1, hi: int | None = None, *, vtab: np.ndarray | None = None, nfb: int = 1,
               learn: bool = False, iteration: int = 1, seeds=(12345678, 87654321), generator: int = 1,
               threads: int | None = None):
    """``adjoint`` with the control variate: every segment's score weighted
    by A - vtab[cell, frequency bin] (vtab: [ncell*nfb], cell-major; None =
    no baseline).  Returns (grad, L, vsum, vcnt); with learn=True vsum/vcnt
    hold the summed A and the count per (cell, bin) at segment starts."""
    lib = load()
    hi = np_total if hi is None else hi
    threads = threads or os.cpu_count() or 1
    c = bundle.config
    ncell = c.nrg * c.ntg * c.npg
    lp = np.ascontiguousarray(lam_psed, dtype=np.float64)
    li = None if lam_img is None else np.ascontiguousarray(lam_img, dtype=np.float64)
    vt = None if vtab is None else np.ascontiguousarray(vtab, dtype=np.float64)
    nv = ncell * abs(nfb) * (4 if nfb < 0 else 1)
    if vt is not None and vt.size != nv:
        raise ValueError("vtab must hold ncell*nfb values")
    grad = np.zeros(ncell * 10, np.float64)
    vs = np.zeros(nv, np.float64) if learn else None
    vc = np.zeros(nv, np.float64) if learn else None
    obj = C.c_double(0.0)
    D = C.POINTER(C.c_double)
    P = (lambda a: a.ctypes.data_as(D) if a is not None else None)
    rc = lib.oracle_adjoint_cv(C.byref(bundle.config), C.byref(bundle.grid), C.byref(bundle.tables), np_total, lo,
                               hi, iteration, seeds[0], seeds[1], generator, threads, lp.ctypes.data_as(D), P(li),
                               grad.ctypes.data_as(D), C.byref(obj), P(vt), nfb, P(vs), P(vc))
    if rc != 0:
        raise RuntimeError(f"oracle_adjoint_cv failed with code {rc}")
    return grad, obj.value, vs, vc


def rep_draine(bundle: abi.Bundle, im: int, n: int, seeds=(12345678, 87654321)) -> np.ndarray:
    """n small-grain re-emission frequencies [eV] from row `im` of the
    Draine spectra (rep_draine_new.f90), one random stream."""
    lib = load()
    out = np.empty(n, np.float64)
    rc = lib.oracle_rep_draine(C.byref(bundle.tables), im, n, seeds[0], seeds[1],
                               out.ctypes.data_as(C.POINTER(C.c_double)))
    if rc != 0:
        raise RuntimeError(f"oracle_rep_draine failed with code {rc}")
    return out


def setemiss(nudust, kappad, adust, nlambda, nT: int = 500, nnu: int = 513, ndg: int | None = None,
             threads: int | None = None) -> dict:
    """Emission tables of the reference's setemiss (dust_5.f90:486-699) from
    dust tables in the engine layout (nudust/kappad/adust: Fortran
    (nlammax, nopac), descending nu per column; nlambda: [nopac]).  Species
    with index > ndg are gas opacities (Planck mean smoothed); default: all
    dust.  Returns lTint, Tint, nuint, kapint (Fortran (nT, nnu, nopac),
    normalised cumulative), kappap, kappar (Fortran (nT, nopac)) and the
    number of qsimp integrals that hit the 20-level limit."""
    lib = load()
    nl = np.ascontiguousarray(nlambda, dtype=np.int32)
    nopac = nl.size
    nud = np.ascontiguousarray(nudust, dtype=np.float64)
    nlammax = nud.size // nopac
    kd = np.ascontiguousarray(kappad, dtype=np.float64)
    ad = np.ascontiguousarray(adust, dtype=np.float64)
    out = dict(lTint=np.zeros(nT), Tint=np.zeros(nT), nuint=np.zeros(nnu), kapint=np.zeros(nT * nnu * nopac),
               kappap=np.zeros(nT * nopac), kappar=np.zeros(nT * nopac))
    miss = C.c_int64(0)
    D = C.POINTER(C.c_double)
    rc = lib.oracle_setemiss(nopac, nopac if ndg is None else ndg, nlammax, nl.ctypes.data_as(C.POINTER(C.c_int32)),
                             nud.ctypes.data_as(D), kd.ctypes.data_as(D), ad.ctypes.data_as(D), nT, nnu,
                             *(out[k].ctypes.data_as(D) for k in ("lTint", "Tint", "nuint", "kapint", "kappap",
                                                                 "kappar")),
                             C.byref(miss), threads or os.cpu_count() or 1)
    if rc != 0:
        raise RuntimeError(f"oracle_setemiss failed ({rc})")
    out["qsimp_misses"] = int(miss.value)
    return out



def diskflux(tal, np_total: int, ltot_lsol: float, nmu: int, nph: int, ipeel: int, imcube: bool) -> dict:
    """diskflux (flux_test.f90:14-82) on the REAL tally arrays of `tal`
    (float32, as the download gives them), in the reference's FP32 order of
    operations: numpy float32 arithmetic is IEEE single precision without
    fused operations, like the Fortran REAL expressions.  Returns the
    normalised arrays by name."""
    f32 = np.float32
    out = {}
    rnorm = f32(float(np_total) / float(nmu) / float(nph) / ltot_lsol)
    inorm = f32(float(np_total) / ltot_lsol)
    si, nums = tal["si"].astype(f32), tal["nums"].astype(f32)
    big = nums > f32(1.0)
    with np.errstate(all="ignore"):
        for k in ("si", "sq", "su", "sv"):
            x, x2 = tal[k].astype(f32), tal[k + "2"].astype(f32)
            e = np.sqrt((x2 - x ** 2 / nums) / (nums - f32(1.0)) * nums) / si
            if k == "si":
                e = e + f32(1.0) / nums
            out[k + "2"] = np.where(big, e, f32(0.0)).astype(f32)
            out[k] = (x / rnorm).astype(f32)
        ave = tal["aveinc"].astype(f32)
        out["aveinc"] = np.where(big, ave / nums, ave).astype(f32)
        out["nums"] = nums
        if ipeel == 1:
            numt = tal["numt"].astype(f32)
            bigt = numt > f32(1.0)
            for k in ("ti", "tq", "tu", "tv"):
                x, x2 = tal[k].astype(f32), tal[k + "2"].astype(f32)
                e = np.sqrt((x2 * numt / x ** 2 - f32(1.0)) / (numt - f32(1.0)))
                out[k + "2"] = np.where(bigt, e, f32(0.0)).astype(f32)
                out[k] = (x / inorm).astype(f32)
            out["numt"] = numt
            if imcube:
                for k in ("image_m_i", "image_m_q", "image_m_u", "image_m_v"):
                    if k in tal.arrays:
                        out[k] = (tal[k].astype(f32) / inorm).astype(f32)
    return out
