"""Host-side mirror of the reference's ``disk`` / Lucy-iteration interface.

``Engine`` drives the CUDA engine through its C ABI (``libmcrt_b200.so``,
include/mcrt_b200.h) exactly as the Fortran driver would through
``iso_c_binding``:

* ``Engine.disk(converge, iteration, i1)`` is ``subroutine disk``
  (newdisktherm_5_fuv.f90:1-663): reset tallies, run the packet loop on the
  GPU, download the reduced tallies, update the dust temperature (``tfinal``)
  and return the new ``converge`` flag;
* ``lucy_iterations`` is the temperature loop of newtts.f90:225-256.

There is no CPU path: if the library cannot be loaded or a call fails, a
``MCRTError`` is raised.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libmcrt_b200.so")
_lib = None


class MCRTError(RuntimeError):
    """A failed C-ABI call; `code` is its MCRT_ERR_* return code."""

    def __init__(self, msg: str, code: int | None = None):
        super().__init__(msg)
        self.code = code


def load_library(path: str = LIB_PATH):
    """Load the engine library; raises if it is missing (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise MCRTError(f"engine library not built: {path} (run __graft_entry__.build())")
    lib = C.CDLL(path)
    P = C.POINTER
    lib.mcrt_create.argtypes = [P(abi.Config), C.c_int, P(C.c_void_p)]
    lib.mcrt_upload_grid.argtypes = [C.c_void_p, P(abi.Grid)]
    lib.mcrt_upload_tables.argtypes = [C.c_void_p, P(abi.Tables)]
    lib.mcrt_set_precision.argtypes = [C.c_void_p, C.c_int32]
    lib.mcrt_set_schedule.argtypes = [C.c_void_p, C.c_int32, C.c_int32]
    lib.mcrt_set_wave_pool.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_int64]
    lib.mcrt_reset_tallies.argtypes = [C.c_void_p]
    lib.mcrt_check_grid.argtypes = [P(abi.Config), P(abi.Grid), C.c_char_p, C.c_int32]
    lib.mcrt_check_grid.restype = C.c_int
    lib.mcrt_set_limits.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_double]
    lib.mcrt_set_limits.restype = C.c_int
    lib.mcrt_diskflux.argtypes = [C.c_void_p, C.c_int64, C.c_double, C.c_int32, P(abi.Tallies)]
    lib.mcrt_diskflux.restype = C.c_int
    lib.mcrt_run_iteration.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_int32, C.c_int32,
                                       C.c_int32, C.c_int32, C.c_int32]
    lib.mcrt_download_tallies.argtypes = [C.c_void_p, P(abi.Tallies)]
    lib.mcrt_accumulate_tallies.argtypes = [C.c_void_p, P(abi.Tallies)]
    lib.mcrt_update_temperature.argtypes = [C.c_void_p, C.c_int32, C.c_int32, P(C.c_double), P(C.c_int32),
                                            P(C.c_double)]
    lib.mcrt_enable_packet_log.argtypes = [C.c_void_p, C.c_int64]
    lib.mcrt_download_packet_log.argtypes = [C.c_void_p, P(abi.PacketLog), C.c_int64]
    lib.mcrt_last_kernel_ms.argtypes = [C.c_void_p, P(C.c_double)]
    lib.mcrt_wave_stats.argtypes = [C.c_void_p, P(C.c_double), P(C.c_int64)]
    lib.mcrt_device_tallies_view.argtypes = [C.c_void_p, P(abi.DeviceTallies)]
    lib.mcrt_refresh_diffusion.argtypes = [C.c_void_p]
    lib.mcrt_setdiffus.argtypes = [C.c_void_p, C.c_int32, C.c_double, C.c_double, P(C.c_double), P(C.c_int32),
                                   P(C.c_int32), P(C.c_int64)]
    D = P(C.c_double)
    lib.mcrt_adjoint.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_int32, C.c_int32, C.c_int32,
                                 C.c_int32, D, D, D, D]
    lib.mcrt_mark.argtypes = [C.c_void_p, C.c_int32]
    lib.mcrt_elapsed_ms.argtypes = [C.c_void_p, C.c_int32, C.c_int32, P(C.c_double)]
    lib.mcrt_flush_l2.argtypes = [C.c_void_p]
    lib.mcrt_synchronize.argtypes = [C.c_void_p]
    lib.mcrt_last_error.argtypes = [C.c_void_p]
    lib.mcrt_last_error.restype = C.c_char_p
    lib.mcrt_destroy.argtypes = [C.c_void_p]
    lib.mcrt_destroy.restype = None
    lib.mcrt_version.restype = C.c_char_p
    lib.mcrt_model_density.argtypes = [C.c_int32, P(abi.DensityParams), C.c_int32, C.c_int32, C.c_int32,
                                       P(C.c_double), P(C.c_double), P(C.c_double), P(C.c_double), P(C.c_double),
                                       P(C.c_double)]
    lib.mcrt_set_adjoint_chunk.argtypes = [C.c_void_p, C.c_int64]
    lib.mcrt_set_adjoint_baseline.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int64, C.c_double]
    lib.mcrt_set_wave_loop.argtypes = [C.c_void_p, C.c_int32]
    lib.mcrt_setemiss.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_int32, P(C.c_int32), P(C.c_double),
                                  P(C.c_double), P(C.c_double), C.c_int32, C.c_int32, P(C.c_double), P(C.c_double),
                                  P(C.c_double), P(C.c_double), P(C.c_double), P(C.c_double), P(C.c_int64),
                                  P(C.c_double)]
    lib.mcrt_batch_create.argtypes = [P(C.c_void_p), C.c_int32, P(C.c_void_p)]
    lib.mcrt_batch_run_iteration.argtypes = [C.c_void_p, P(C.c_int64), C.c_int32, C.c_int32, C.c_int32, C.c_int32]
    lib.mcrt_batch_tune.argtypes = [C.c_void_p, C.c_int64, P(C.c_int32)]
    lib.mcrt_batch_set_schedule.argtypes = [C.c_void_p, C.c_int32, C.c_int64]
    lib.mcrt_batch_set_tuning.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32]
    lib.mcrt_batch_last_ms.argtypes = [C.c_void_p, P(C.c_double)]
    lib.mcrt_batch_last_error.argtypes = [C.c_void_p]
    lib.mcrt_batch_last_error.restype = C.c_char_p
    lib.mcrt_batch_destroy.argtypes = [C.c_void_p]
    lib.mcrt_batch_destroy.restype = None
    for name in ("mcrt_create", "mcrt_upload_grid", "mcrt_upload_tables", "mcrt_set_precision", "mcrt_set_schedule",
                 "mcrt_set_wave_pool", "mcrt_reset_tallies", "mcrt_run_iteration", "mcrt_download_tallies",
                 "mcrt_accumulate_tallies", "mcrt_update_temperature", "mcrt_enable_packet_log",
                 "mcrt_download_packet_log", "mcrt_last_kernel_ms", "mcrt_wave_stats", "mcrt_mark", "mcrt_elapsed_ms",
                 "mcrt_device_tallies_view", "mcrt_refresh_diffusion", "mcrt_setdiffus", "mcrt_adjoint",
                 "mcrt_flush_l2", "mcrt_synchronize", "mcrt_batch_create", "mcrt_batch_run_iteration",
                 "mcrt_batch_tune", "mcrt_batch_set_schedule", "mcrt_batch_set_tuning", "mcrt_batch_last_ms",
                 "mcrt_setemiss", "mcrt_set_adjoint_chunk", "mcrt_set_adjoint_baseline", "mcrt_set_wave_loop", "mcrt_model_density"):
        getattr(lib, name).restype = C.c_int
    _lib = lib
    return lib


def setemiss(nudust, kappad, adust, nlambda, ndg: int | None = None, nT: int = 500, nnu: int = 513,
             device: int = 0) -> dict:
    """The reference's emission tables (dustinit grids and setemiss,
    dust_5.f90:486-699) built on the GPU (C ABI ``mcrt_setemiss``).

    nudust/kappad/adust: Fortran (nlammax, nopac) as in ``mcrt_tables``
    (nu strictly decreasing per species); nlambda: [nopac]; species above
    `ndg` (default: none) are gas opacities.  Returns lTint, Tint, nuint,
    kapint (nT*nnu*nopac, Fortran), kappap, kappar (nT*nopac), the count of
    qsimp integrals that hit the level limit and the kernel time [ms]."""
    lib = load_library()
    nl = np.ascontiguousarray(nlambda, dtype=np.int32)
    nopac = nl.size
    nud = np.ascontiguousarray(nudust, dtype=np.float64)
    kd = np.ascontiguousarray(kappad, dtype=np.float64)
    ad = np.ascontiguousarray(adust, dtype=np.float64)
    nlammax = nud.size // nopac
    out = dict(lTint=np.zeros(nT), Tint=np.zeros(nT), nuint=np.zeros(nnu), kapint=np.zeros(nT * nnu * nopac),
               kappap=np.zeros(nT * nopac), kappar=np.zeros(nT * nopac))
    miss = C.c_int64(0)
    ms = C.c_double(0.0)
    D = C.POINTER(C.c_double)
    rc = lib.mcrt_setemiss(device, nopac, nopac if ndg is None else ndg, nlammax,
                           nl.ctypes.data_as(C.POINTER(C.c_int32)), nud.ctypes.data_as(D), kd.ctypes.data_as(D),
                           ad.ctypes.data_as(D), nT, nnu,
                           *(out[k].ctypes.data_as(D) for k in ("lTint", "Tint", "nuint", "kapint", "kappap",
                                                               "kappar")),
                           C.byref(miss), C.byref(ms))
    if rc != 0:
        raise MCRTError(f"mcrt_setemiss failed (code {rc}): {lib.mcrt_last_error(None).decode()}")
    out["qsimp_misses"] = int(miss.value)
    out["device_ms"] = ms.value
    return out


def check_grid(model) -> tuple:
    """mcrt_check_grid on a model's arrays (host only, no device): the
    return code and the message naming the first bad entry."""
    lib = load_library()
    b = abi.Bundle(model)
    msg = C.create_string_buffer(256)
    rc = lib.mcrt_check_grid(C.byref(b.config), C.byref(b.grid), msg, 256)
    return rc, msg.value.decode()


def density_params(w) -> "abi.DensityParams":
    """mcrt_density_params of a model.Workload (lengths to stellar radii)."""
    autors = 214.94 / w.rstar
    return abi.DensityParams(rstar=w.rstar, autors=autors, rddust=w.rddust_au * autors, rmax=w.rmax_au * autors,
                             rmaxd=w.rmaxd_au * autors, massd=w.massd, a_exp=w.a_exp, b_exp=w.b_exp,
                             h100_au=w.h100_au, rate=w.rate, rc=w.rc_au * autors, massc=w.massc, rhoamb=w.rhoamb,
                             thet1_deg=w.thet1_deg, ex1=w.ex1, rhoconst1=w.rhoconst1)


def model_density(model, device: int = 0, derivatives: bool = True):
    """The model's density grid built on the GPU (C ABI mcrt_model_density)
    from its Workload parameters and walls: (densarr [ncell*10] Fortran,
    vcell [ncell], dlog_disk or None).  dlog_disk is Fortran
    (nrg-1, ntg-1, 3): d log rho_disk / d (log Mdisk, b, log h100), analytic."""
    lib = load_library()
    w = model.w
    nrg, ntg, npg = w.nrg, w.ntg, w.npg
    prm = density_params(w)
    D = C.POINTER(C.c_double)
    rarr = np.ascontiguousarray(model.grid["rarr"], dtype=np.float64)
    thetarr = np.ascontiguousarray(model.grid["thetarr"], dtype=np.float64)
    clump = None
    if w.clump_seed is not None:
        clump = np.asfortranarray(model._clump_field(nrg - 1, ntg - 1, max(npg - 1, 1))).ravel(order="F")
    dens = np.zeros(nrg * ntg * npg * 10)
    vcell = np.zeros(nrg * ntg * npg)
    dlog = np.zeros((nrg - 1) * (ntg - 1) * 3) if derivatives else None
    rc = lib.mcrt_model_density(device, C.byref(prm), nrg, ntg, npg, rarr.ctypes.data_as(D),
                                thetarr.ctypes.data_as(D), clump.ctypes.data_as(D) if clump is not None else None,
                                dens.ctypes.data_as(D), vcell.ctypes.data_as(D),
                                dlog.ctypes.data_as(D) if dlog is not None else None)
    if rc != 0:
        raise MCRTError(f"mcrt_model_density failed (code {rc}): {lib.mcrt_last_error(None).decode()}")
    return dens, vcell, dlog


def with_setemiss_tables(model, ndg: int | None = None, device: int = 0):
    """Replace the model's emission tables by the reference's setemiss
    tables built on the GPU (the model generator uses its own quadrature)."""
    t = model.tables
    r = setemiss(t["nudust"], t["kappad"], t["adust"], t["nlambda"], ndg=ndg, device=device)
    for k in ("lTint", "Tint", "nuint", "kapint", "kappap", "kappar"):
        t[k] = r[k]
    model.config["nT"] = r["lTint"].size
    model.config["nnu"] = r["nuint"].size
    return model


class Engine:
    """One GPU context holding one model (the state ``disk`` reads)."""

    def __init__(self, model, device: int = 0, precision: str = "fp64"):
        self.lib = load_library()
        self.model = model
        self.bundle = abi.Bundle(model)
        self.cfg = self.bundle.config
        ctx = C.c_void_p()
        self._check(self.lib.mcrt_create(C.byref(self.cfg), device, C.byref(ctx)), ctx)
        self.ctx = ctx
        self.set_precision(precision)
        self.upload_grid()
        self.upload_tables()
        self.tdave = model.grid["tdust"].copy()
        self.sig = np.full(3, np.nan)

    # ------------------------------------------------------------ plumbing
    def _check(self, rc, ctx=None):
        if rc != 0:
            c = ctx if ctx is not None else self.ctx
            msg = self.lib.mcrt_last_error(c).decode() if c else ""
            raise MCRTError(f"mcrt call failed (code {rc}): {msg}", rc)

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.mcrt_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_precision(self, precision: str):
        mode = {"fp64": abi.PREC_FP64, "mixed": abi.PREC_MIXED}[precision]
        self._check(self.lib.mcrt_set_precision(self.ctx, mode))
        self.precision = precision

    def set_schedule(self, schedule: str = "wave", event_batch: int | None = None):
        """Kernel schedule: "packet" (one thread per packet), "warp" (lockstep
        lanes, batched events) or "wave" (walk / event kernels over a pool of
        in-flight packets).  `event_batch`: warp schedule -- lanes waiting
        before events run (default 16); wave -- idle lanes before a walk
        warp takes new walks (default 4)."""
        mode = {"packet": 0, "warp": 1, "wave": 2}[schedule]
        if event_batch is None:
            event_batch = 4 if schedule == "wave" else 16
        self._check(self.lib.mcrt_set_schedule(self.ctx, mode, event_batch))
        self.schedule = schedule

    def set_limits(self, walk_crossings: int = 0, waves: int = 0, geom_fraction: float = 1e-6):
        """Watchdogs (mcrt_set_limits): crossings per walk before a packet is
        dropped as a geometry failure, waves per wavefront loop before a run
        returns MCRT_ERR_TIMEOUT, and the fraction of lost packets above
        which a run returns MCRT_ERR_GEOM (0 / 0: the defaults)."""
        self._check(self.lib.mcrt_set_limits(self.ctx, walk_crossings, waves, geom_fraction))

    def set_wave_pool(self, slots: int = 1 << 21, peel_jobs: int = 0, tail_packets: int = -1):
        """Wavefront schedule sizes: in-flight packet slots, peel-off job
        queue capacity (0: default) and the live-packet count at which one
        tail launch finishes the iteration (<0: default, 0: never)."""
        self._check(self.lib.mcrt_set_wave_pool(self.ctx, int(slots), int(peel_jobs), int(tail_packets)))

    def set_wave_loop(self, device: bool = True):
        """Wavefront loop driven by the device (one graph launch per
        iteration) or by the host (a synchronisation after every walk
        launch); C ABI ``mcrt_set_wave_loop``."""
        self._check(self.lib.mcrt_set_wave_loop(self.ctx, 1 if device else 0))

    def upload_grid(self):
        self.bundle = abi.Bundle(self.model)
        self._check(self.lib.mcrt_upload_grid(self.ctx, C.byref(self.bundle.grid)))

    def upload_tables(self):
        self._check(self.lib.mcrt_upload_tables(self.ctx, C.byref(self.bundle.tables)))

    def reset_tallies(self):
        self._check(self.lib.mcrt_reset_tallies(self.ctx))

    def run(self, np_total: int, lo: int = 1, hi: int | None = None, *, iteration: int = 1, ipeel: int = 1,
            seeds=(12345678, 87654321), generator: int = 1):
        hi = np_total if hi is None else hi
        self._check(self.lib.mcrt_run_iteration(self.ctx, np_total, lo, hi, iteration, ipeel,
                                                seeds[0], seeds[1], generator))

    def kernel_ms(self) -> float:
        v = C.c_double()
        self._check(self.lib.mcrt_last_kernel_ms(self.ctx, C.byref(v)))
        return v.value

    def wave_stats(self) -> dict:
        """Per-kernel device time and counts of the last wavefront run."""
        ms = (C.c_double * 4)()
        n = (C.c_int64 * 6)()
        self._check(self.lib.mcrt_wave_stats(self.ctx, ms, n))
        names = ("walk", "event", "tail", "peel")
        out = {f"{k}_ms": ms[i] for i, k in enumerate(names)}
        out.update({f"{k}_launches": n[i] for i, k in enumerate(names)})
        out["walks"] = n[4]
        out["walk_crossings"] = n[5]
        return out

    def mark(self, slot: int):
        self._check(self.lib.mcrt_mark(self.ctx, slot))

    def elapsed_ms(self, a: int, b: int) -> float:
        v = C.c_double()
        self._check(self.lib.mcrt_elapsed_ms(self.ctx, a, b, C.byref(v)))
        return v.value

    def flush_l2(self):
        self._check(self.lib.mcrt_flush_l2(self.ctx))

    def synchronize(self):
        self._check(self.lib.mcrt_synchronize(self.ctx))

    def download(self, images: bool = True) -> abi.TallyArrays:
        tal = abi.TallyArrays(self.cfg, images=images)
        self._check(self.lib.mcrt_download_tallies(self.ctx, C.byref(tal.struct)))
        return tal

    def diskflux(self, np_total: int, ltot_lsol: float, ipeel: int = 1, images: bool = True) -> abi.TallyArrays:
        """``subroutine diskflux`` (flux_test.f90): the tallies with the
        reference's output normalisation and error arrays, computed on the
        device (mcrt_diskflux)."""
        tal = abi.TallyArrays(self.cfg, images=images)
        self._check(self.lib.mcrt_diskflux(self.ctx, np_total, ltot_lsol, ipeel, C.byref(tal.struct)))
        return tal

    def accumulate(self, tal: abi.TallyArrays):
        """Add host tallies (e.g. the sum over ranks) into the device tallies."""
        self._check(self.lib.mcrt_accumulate_tallies(self.ctx, C.byref(tal.struct)))

    def device_tallies(self) -> abi.DeviceTallies:
        """Device addresses and lengths of the tally segments (in-place all-reduce)."""
        v = abi.DeviceTallies()
        self._check(self.lib.mcrt_device_tallies_view(self.ctx, C.byref(v)))
        return v

    def adjoint(self, np_total: int, lam_psed, lam_img=None, lo: int = 1, hi: int | None = None, *,
                iteration: int = 1, seeds=(12345678, 87654321), generator: int = 1):
        """Path-replay adjoint of L = sum lam_psed*ti + sum lam_img*image_m_i:
        returns (dL/dlog(rho) as [ncell*10] Fortran (nrg,ntg,npg,10), L)."""
        hi = np_total if hi is None else hi
        c = self.cfg
        lp = np.ascontiguousarray(lam_psed, dtype=np.float64)
        li = None if lam_img is None else np.ascontiguousarray(lam_img, dtype=np.float64)
        grad = np.zeros(c.nrg * c.ntg * c.npg * 10, np.float64)
        obj = C.c_double(0.0)
        D = C.POINTER(C.c_double)
        self._check(self.lib.mcrt_adjoint(self.ctx, np_total, lo, hi, iteration, seeds[0], seeds[1], generator,
                                          lp.ctypes.data_as(D), li.ctypes.data_as(D) if li is not None else None,
                                          grad.ctypes.data_as(D), C.byref(obj)))
        return grad, obj.value

    def set_adjoint_chunk(self, packets: int):
        """Packets per adjoint chunk (forward, sort and replay per chunk;
        gradients and objective summed)."""
        self._check(self.lib.mcrt_set_adjoint_chunk(self.ctx, int(packets)))

    def set_adjoint_baseline(self, nfb: int = 10, ndir: int = 4, pilot_packets: int = 1_000_000,
                             min_count: float = 16.0):
        """Control variate of the adjoint's replay (C ABI
        ``mcrt_set_adjoint_baseline``): the mean future contribution per
        (cell, frequency bin, direction class), learned from a pilot replay
        of `pilot_packets` packets on another generator, is subtracted from
        each segment's weight.  ``nfb=0`` switches it off."""
        self._check(self.lib.mcrt_set_adjoint_baseline(self.ctx, int(nfb), int(ndir), int(pilot_packets),
                                                       float(min_count)))

    def refresh_diffusion(self):
        """Diffusion-cell temperatures of the last run from the (reduced) counts."""
        self._check(self.lib.mcrt_refresh_diffusion(self.ctx))

    def setdiffus(self, iteration: int, tdave=None, outputs: bool = True):
        """setdiffus(iter) and gridset's tdust reset on the device
        (mcrt_setdiffus), from ``tdave`` (default: the engine's current
        temperature); returns (diffus, diffdir, dcount) as Fortran-order
        flat arrays, or None with ``outputs=False`` (the call then returns
        without waiting for the device).  The disk mass and outer radius
        come from the model."""
        w = self.model.w
        td = np.ascontiguousarray(self.tdave if tdave is None else tdave, dtype=np.float64)
        n = td.size
        I = C.POINTER(C.c_int32)
        args = (self.ctx, iteration, float(w.massd), float(w.rmaxd_au * self.model.config["autors"]),
                td.ctypes.data_as(C.POINTER(C.c_double)))
        if not outputs:
            self._check(self.lib.mcrt_setdiffus(*args, None, None, None))
            return None
        dif = np.zeros(n, np.int32)
        ddir = np.zeros(n, np.int32)
        cnt = C.c_int64(0)
        self._check(self.lib.mcrt_setdiffus(*args, dif.ctypes.data_as(I), ddir.ctypes.data_as(I), C.byref(cnt)))
        return dif, ddir, int(cnt.value)

    def enable_packet_log(self, n: int):
        self._check(self.lib.mcrt_enable_packet_log(self.ctx, n))

    def packet_log(self, n: int):
        log = abi.packet_log_array(n)
        self._check(self.lib.mcrt_download_packet_log(self.ctx, log, n))
        return log

    def update_temperature(self, nphot: int, iteration: int, converge: int = 0):
        td = np.ascontiguousarray(self.tdave, dtype=np.float64).copy()
        conv = C.c_int32(converge)
        sig = np.zeros(3, np.float64)
        self._check(self.lib.mcrt_update_temperature(self.ctx, nphot, iteration,
                                                     td.ctypes.data_as(C.POINTER(C.c_double)), C.byref(conv),
                                                     sig.ctypes.data_as(C.POINTER(C.c_double))))
        self.tdave = td
        self.sig = sig
        return td, bool(conv.value), sig

    # --------------------------------------------------- reference interface
    def disk(self, converge: str, iteration: int, i1: int, np_total: int, *, ipeel: int = 0,
             generator: int = 1):
        """``subroutine disk(converge,iter,i1)`` for one GPU.

        Runs np_total packets (the packet loop), leaves the reduced tallies in
        ``self.tallies`` and updates the temperature with ``tfinal``;
        returns the new ``converge`` ('yes'/'no').  A model with the
        diffusion treatment first recomputes its diffusion region from the
        current temperature, as gridset does every iteration
        (gridset_5_model13new.f90:1842-1866, ``setdiffus``).
        """
        if self.model.config.get("diffusion") and iteration >= 1:
            self.setdiffus(iteration, outputs=False)
        self.reset_tallies()
        self.run(np_total, iteration=iteration, ipeel=ipeel, seeds=(12345678 - i1 if i1 else 12345678, 87654321),
                 generator=generator)
        self.tallies = self.download(images=bool(ipeel))
        _, conv, _ = self.update_temperature(np_total, iteration, 1 if converge == "yes" else 0)
        return "yes" if conv else "no"


def lucy_iterations(engine: Engine, np_total: int, n_iter: int, n_iter_min: int = 0):
    """The Lucy loop of newtts.f90:225-256 (no peel-off during iterations)."""
    converge = "no"
    it = 0
    history = []
    while converge == "no":
        it += 1
        converge = engine.disk(converge, it, 0, np_total, ipeel=0)
        history.append(engine.sig.copy())
        if it < n_iter_min:
            converge = "no"
        if it >= n_iter:
            converge = "yes"
    return it, history
