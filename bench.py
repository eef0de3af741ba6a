"""Benchmark: photon packets/s of the B200 engine on the 2-D young-star model.

Workload (the configuration the headline metric is quoted on): the 2-D disk +
Ulrich envelope + bipolar cavity model (nr=100 x ntheta=99 x nphi=1 cells,
4000 K / 2 Rsun star, Mdisk=0.01 Msun, 100 log wavelengths 0.1-3000 um),
run as Lucy iterations of the reference's ``disk`` routine.  One step is one
iteration: the diffusion region of the current temperature (``setdiffus``,
as gridset reruns it every iteration), the packet loop over ``--packets``
packets per GPU (emission, cell walk, scattering, absorption + Lucy
reemission, exit binning) and the device temperature update (``tfinal``).
Inputs are synthetic (seeded generator, no reference parameter files exist
here).

value : packets/s of the whole job (all ranks), device-timed between CUDA
        events on the engine's stream, max over ranks;
e2e   : the same through the public C ABI with host buffers: grid upload
        (host->device), iteration, tally + temperature download
        (device->host) inside the timed region.

``--impl reference`` times the CPU restatement of the reference's packet
loop (the oracle; the Fortran itself cannot be built here) on all host
cores for a bounded sample of the same workload.

Further keys of the line, each measured once after the timed steps:

* ``roofline`` (the walk kernel against HBM) and ``roofline_compute``
  (against the FP64 rate);
* the FP64 build and the plain per-thread FP64 path (``fp64_value``,
  ``fp64_plain``);
* the peeled imaging iteration and the mixed-vs-FP64 errors;
* ``gradient``: the path-replay adjoint of the peeled SED and images;
* ``clumpy_3d``: the 3-D clumpy model with tabulated Mueller matrices,
  peeled, on a sample of its 1e9-packet run;
* ``setemiss``: the emission tables built on the GPU;
* ``batch``: the 64-model sweep, sharded over the ranks under torchrun;
* ``cpu_baseline``.

Flags switch the sections off (``--grad-packets 0``, ``--clumpy-packets 0``,
``--batch-models 0``, ``--no-compare``, ``--no-cpu-baseline``).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "photon packets/s (1 B200): mixed vs FP64 plain at equal SED error; grad time"
UNIT = "packets/s"


def _peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {"hbm_gbs": 6650.0, "_fallback": True}


class Clocks:
    """nvidia-smi sampler for the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self._p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                        "--format=csv,noheader,nounits", "-lms", "200"],
                                       stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self._p = None
        return self

    def _read(self):
        for line in self._p.stdout:
            if self._stop.is_set():
                break
            self.samples.append([s.strip() for s in line.split(",")])

    def __exit__(self, *a):
        self._stop.set()
        if self._p:
            self._p.terminate()
            try:
                self._p.wait(timeout=5)
            except Exception:
                self._p.kill()

    def summary(self):
        import statistics
        sm = [float(s[0]) for s in self.samples if len(s) >= 7 and s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if len(s) >= 7 and s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            if len(s) >= 7:
                for k, n in enumerate(names):
                    if s[3 + k].lower().startswith("active"):
                        reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def build_model(args):
    """The 2-D workload at its converged Lucy temperature (the state a Lucy
    sequence settles in; committed with the package), with the reference's
    default diffusion treatment of the optically thick disk interior
    (DIFFUSION=YES, tts_mod_5.f90:33).  Every arm -- the GPU steps, the
    CPU baseline and the reference arm -- starts from this same state."""
    from src3_mpi_cfitsio_b200 import model
    return model.with_velocities(model.reference_2d_converged())


def algorithmic_bytes(c: dict) -> float:
    """Algorithmic bytes of one transport launch: 16 B per walk crossing
    (density + species record 8 B, FP64 dtauabs update 8 B), 8 B per
    peel-off crossing, 64 B per interaction (opacity row 32 B + packet
    state 32 B), 16 B per SED / peel-off bin (4 x FP32 Stokes)."""
    return (16.0 * c["crossings"] + 8.0 * c["peel_cross"] + 64.0 * c["interactions"] +
            16.0 * (c["exited"] + c["peel_binned"]))


def _errors(a, b):
    """Relative L1 distance of tally b from tally a (per-bin SED, images)."""
    import numpy as np
    out = {}
    for k in ("si", "ti", "image_m_i", "image_m_q"):
        if k in a.arrays and k in b.arrays:
            x = a[k].astype(np.float64)
            y = b[k].astype(np.float64)
            den = np.abs(x).sum()
            if den > 0:
                out[k] = float(np.abs(y - x).sum() / den)
    return out


def bench_clumpy(args, dev):
    """3-D clumpy model (nr=200, ntheta=199, nphi=64, fractal clumps, tabulated
    S11-S44 scattering matrices), mixed precision, peeled iteration with
    201x201 Stokes images at 20 wavelengths and 20 inclinations: device
    packets/s on a sample of the 1e9-packet run."""
    from src3_mpi_cfitsio_b200 import model
    from src3_mpi_cfitsio_b200.engine import Engine
    m = model.with_diffusion(model.warm(model.with_mueller(model.clumpy_3d())))
    eng = Engine(m, device=dev, precision="mixed")
    eng.set_schedule("wave")
    n = args.clumpy_packets
    eng.reset_tallies()
    eng.run(max(n // 10, 1000), iteration=1, ipeel=1)          # warm
    eng.reset_tallies()
    eng.flush_l2()
    eng.run(n, iteration=2, ipeel=1)
    ms = eng.kernel_ms()
    ws = eng.wave_stats()
    c = eng.download(images=False).counters()
    # the FP64 build on a smaller sample of the same iteration
    n64 = max(n // 5, 1000)
    eng.set_precision("fp64")
    eng.reset_tallies()
    eng.flush_l2()
    eng.run(n, 1, n64, iteration=2, ipeel=1)
    ms64 = eng.kernel_ms()
    eng.close()
    return {"workload": "3-D clumpy (nr=200, ntheta=199, nphi=64; fractal dim 2.6, 50% mass in clumps), tabulated "
                        "Mueller matrices, 201x201 images x 4 Stokes x 20 wavelengths x 20 inclinations, peel-off on",
            "packets": n, "precision": "mixed", "packets_per_s": n / (ms / 1e3),
            "seconds_for_1e9": 1e9 / (n / (ms / 1e3)),
            "kernels_ms": {k: ws[f"{k}_ms"] for k in ("walk", "event", "tail", "peel")},
            "fp64_packets": n64, "fp64_packets_per_s": n64 / (ms64 / 1e3),
            "mixed_over_fp64": (n / ms) / (n64 / ms64),
            "crossings_per_packet": c["crossings"] / n, "peel_crossings_per_packet": c["peel_cross"] / n}


def bench_velocity(args, dev):
    """What the velocity terms of tfinal (dusttemp_5.f90:42-53, the infall
    field of the envelope) do to the temperatures: one iteration's tallies,
    tfinal with the field and without it on the same dtauabs, iteration 5
    (20 passes, the last 10 averaged)."""
    import copy
    import numpy as np
    from src3_mpi_cfitsio_b200.engine import Engine
    m = build_model(args)
    rest = copy.deepcopy(m)
    for k in ("vrarr", "vthetarr", "divvarr"):
        del rest.grid[k]
    n = 10_000_000
    ev = Engine(m, device=dev, precision="mixed")
    ev.reset_tallies()
    ev.run(n, iteration=5, ipeel=0)
    tal = ev.download(images=False)
    t0 = time.perf_counter()
    tv, _, _ = ev.update_temperature(n, 5)
    tv_s = time.perf_counter() - t0
    er = Engine(rest, device=dev, precision="mixed")
    er.reset_tallies()
    er.accumulate(tal)
    t0 = time.perf_counter()
    tr, _, _ = er.update_temperature(n, 5)
    tr_s = time.perf_counter() - t0
    ev.close()
    er.close()
    env = (m.dens4()[..., 2] > 0).ravel(order="F") & (tr > 2.0 / 11605.0)
    rel = np.abs(tv[env] / tr[env] - 1.0)
    return {"packets": n, "iteration": 5, "envelope_cells": int(env.sum()),
            "rel_change_median": float(np.median(rel)), "rel_change_max": float(rel.max()),
            "tfinal_seconds_with_velocity": tv_s, "tfinal_seconds_at_rest": tr_s}


def bench_setemiss(args, dev):
    """The emission tables of dustinit/setemiss (dust_5.f90:486-699) built on
    the GPU: the model's 8 dust species, and 187 species (the reference's
    opacity count: its dust plus gas tables) made by perturbing them."""
    import numpy as np

    from src3_mpi_cfitsio_b200 import model
    from src3_mpi_cfitsio_b200.engine import setemiss
    t = model.reference_2d().tables
    nl = np.asarray(t["nlambda"])
    nlm = t["nudust"].size // nl.size
    out = {}
    for nsp in (nl.size, 187):
        reps = -(-nsp // nl.size)
        scale = np.repeat(1.0 + 0.01 * np.arange(reps * nl.size), nlm)[:nsp * nlm]
        kd = np.tile(t["kappad"], reps)[:nsp * nlm] * scale
        r = setemiss(np.tile(t["nudust"], reps)[:nsp * nlm], kd, np.tile(t["adust"], reps)[:nsp * nlm],
                     np.tile(nl, reps)[:nsp], device=dev)
        t0 = time.perf_counter()
        r = setemiss(np.tile(t["nudust"], reps)[:nsp * nlm], kd, np.tile(t["adust"], reps)[:nsp * nlm],
                     np.tile(nl, reps)[:nsp], device=dev)
        out[f"species_{nsp}"] = {"device_ms": r["device_ms"], "wall_ms": 1e3 * (time.perf_counter() - t0),
                                 "qsimp_misses": r["qsimp_misses"]}
    out["grid"] = "nT=500 temperatures x nnu=513 frequency intervals, two qsimp integrals each"
    return out


def bench_batch(args, dev, rank=0, world=1, allreduce=None):
    """Batched sweep: `--batch-models` seeded uneven models (nr 50-200,
    ntheta 49-199, nphi 1-32; Mdisk, Mdot, cavity angle and wavelength set
    drawn from the seed), `--batch-packets` packets each, mixed precision,
    one Lucy iteration per CUDA-graph launch, schedule and queue sizes from
    the autotuner.  Under torchrun the models are sharded whole over the
    ranks (dist.shard_models, no exchange) and the time is the maximum over
    ranks.  Compared with the same models run one after another (Engine.run,
    wavefront schedule) on a sample of 8 of rank 0's models."""
    import numpy as np

    from src3_mpi_cfitsio_b200 import dist, model
    from src3_mpi_cfitsio_b200.batch import Batch
    from src3_mpi_cfitsio_b200.engine import Engine
    nmod, n = args.batch_models, args.batch_packets
    works = model.batch_workloads(nmod)
    mine = dist.shard_models([w.nrg + w.ntg + w.npg for w in works], world)[rank]   # ~crossings per packet
    models = [model.with_diffusion(model.warm(model.batch_model(works[i]))) for i in mine]
    engines = [Engine(m, device=dev, precision="mixed") for m in models]
    ms = 0.0
    tuned = None
    pk = 0
    if engines:
        b = Batch(engines)
        tuned = b.tune(args.batch_tune_packets)
        b.run_iteration([n] * len(engines), iteration=1)          # capture + warm
        b.run_iteration([n] * len(engines), iteration=2)
        ms = b.kernel_ms()
        pk = sum(e.download(images=False).counters()["packets"] for e in engines)
        b.close()
    ms_max = float(allreduce(np.array([ms]), "max")[0]) if allreduce else ms
    pk_all = int(allreduce(np.array([float(pk)]), "sum")[0]) if allreduce else pk
    seq_pps = None
    if rank == 0 and engines:
        seq_ms = 0.0
        sample = engines[:min(8, len(engines))]
        for e in sample:
            e.set_schedule("wave")
            e.reset_tallies()
            e.run(n, iteration=2, ipeel=0)
            seq_ms += e.kernel_ms()
        seq_pps = len(sample) * n / (seq_ms / 1e3)
    for e in engines:
        e.close()
    if rank != 0:
        return None
    cells = [(w.nrg - 1) * (w.ntg - 1) * (w.npg - 1) for w in works]
    own = len(mine) * n / (ms / 1e3) if ms > 0 else None
    return {"workload": f"{nmod} uneven models (cells {min(cells)}-{max(cells)}), {n:.0e} packets each, one Lucy "
                        "iteration per graph launch, diffusion on",
            "models": nmod, "packets_per_model": n, "packets_total": pk_all, "precision": "mixed",
            "ranks": world, "models_on_rank0": len(mine),
            "packets_per_s": nmod * n / (ms_max / 1e3), "seconds": ms_max / 1e3,
            "tuning_rank0": tuned,
            "sequential_wave_packets_per_s_rank0": seq_pps,
            "batch_over_sequential_rank0": (own / seq_pps) if (own and seq_pps) else None,
            "sequential_sample": "first 8 of rank 0's models, Engine.run each (host-driven wavefront loop)"}


def run_ours(args, rank, world):
    import numpy as np

    from src3_mpi_cfitsio_b200.engine import Engine

    dev = int(os.environ.get("LOCAL_RANK", 0))
    m = build_model(args)
    eng = Engine(m, device=dev, precision=args.precision)
    eng.set_schedule(args.schedule)
    P = args.packets
    np_total = P * world
    lo, hi = rank * P + 1, (rank + 1) * P
    dist = world > 1
    if dist:
        import torch
        import torch.distributed as tdist

    def allreduce(arr, op="sum"):
        if not dist:
            return arr
        t = torch.from_numpy(np.ascontiguousarray(arr)).cuda(dev)
        tdist.all_reduce(t, op=tdist.ReduceOp.SUM if op == "sum" else tdist.ReduceOp.MAX)
        return t.cpu().numpy()

    def reduce_ranks(e):
        """The rank reduction of the tallies: NCCL all-reduce of the device
        tally buffer in place, then the diffusion refresh from the summed
        counts (newdisktherm_5_fuv.f90:520-604)."""
        if dist:
            from src3_mpi_cfitsio_b200 import dist as mdist
            mdist.allreduce_device_tallies(e, device=dev)
            e.refresh_diffusion()

    # gridset reruns setdiffus at the start of every iteration
    # (gridset_5_model13new.f90:1842-1866): the diffusion region follows tdave
    diffusion = bool(m.config.get("diffusion"))

    def step(it, e, precision=None):
        if diffusion:
            e.setdiffus(it, outputs=False)
        e.reset_tallies()
        e.run(np_total, lo, hi, iteration=it, ipeel=args.ipeel)
        kms = e.kernel_ms()
        reduce_ranks(e)
        e.update_temperature(np_total, it)
        return kms

    # warm-up Lucy iterations (they also bring the temperature toward convergence)
    for w in range(args.warmup):
        step(w + 1, eng)
    eng.synchronize()
    if dist:
        tdist.barrier()
    kernel_ms = []
    with Clocks(dev) as clk:
        eng.flush_l2()
        eng.mark(0)
        for s in range(args.steps):
            it = args.warmup + s + 1
            if diffusion:
                eng.setdiffus(it, outputs=False)
            eng.reset_tallies()
            eng.run(np_total, lo, hi, iteration=it, ipeel=args.ipeel)
            kernel_ms.append(eng.kernel_ms())
            if args.schedule == "wave":
                wave_stats_last = eng.wave_stats()
            reduce_ranks(eng)
            eng.update_temperature(np_total, it)
            if s + 1 < args.steps:
                eng.flush_l2()
        eng.mark(1)
        eng.synchronize()
        ms = eng.elapsed_ms(0, 1)
    tal_last = eng.download(images=bool(args.ipeel))
    counters = tal_last.counters()
    flush_ms = 0.0
    if args.steps > 1:
        eng.mark(2)
        eng.flush_l2()
        eng.mark(3)
        flush_ms = eng.elapsed_ms(2, 3) * (args.steps - 1)
    ms_steps = float(allreduce(np.array([ms - flush_ms]), "max")[0])
    value = np_total * args.steps / (ms_steps / 1e3)

    # ---- end-to-end through the public API with host buffers: per step the
    # driver's grid arrays go up (with the dust temperature of the previous
    # tfinal, as the Fortran driver holds it), the iteration runs, and the
    # tallies and the new temperature come back
    from src3_mpi_cfitsio_b200 import model as mdl
    h2d = sum(m.grid[n].nbytes for n in ("densarr", "findopac", "diffus", "diffdir", "tdust", "vcell"))
    eng.synchronize()
    e2e_steps = []
    for s in range(args.steps):
        it = args.warmup + args.steps + 1 + s
        m.grid["tdust"] = mdl.tdust_from_tdave(m, eng.tdave)
        eng.flush_l2()
        eng.synchronize()
        t0 = time.perf_counter()
        eng.mark(4)
        eng.upload_grid()
        if diffusion:
            eng.setdiffus(it, outputs=False)
        eng.reset_tallies()
        eng.run(np_total, lo, hi, iteration=it, ipeel=args.ipeel)
        reduce_ranks(eng)
        tl = eng.download(images=bool(args.ipeel))
        td, _, _ = eng.update_temperature(np_total, it)
        eng.mark(5)
        eng.synchronize()
        e2e_steps.append(max(eng.elapsed_ms(4, 5), (time.perf_counter() - t0) * 1e3))
    e2e_ms = sum(e2e_steps) / len(e2e_steps)
    d2h = sum(a.nbytes for a in tl.arrays.values()) + td.nbytes
    if diffusion:   # setdiffus: tdave up, the packed flags (int32 per cell) down
        h2d += eng.tdave.nbytes
        d2h += 4 * eng.tdave.size
    e2e_ms = float(allreduce(np.array([e2e_ms]), "max")[0])
    e2e = np_total / (e2e_ms / 1e3)

    # ---- roofline of the dominant kernel (last timed step)
    peaks = _peaks()
    peak = peaks.get("hbm_gbs", 6650.0)
    kernels = None
    traffic = None
    if args.schedule == "wave":
        # wavefront: the walk kernel carries the cell crossings; achieved =
        # 16 B per crossing it stepped / its summed launch time (the same
        # ratio as per launch); traffic = DRAM bytes per walk (ncu capture)
        # x walks per walk launch
        ws = wave_stats_last
        kernels = {k: ws[f"{k}_ms"] for k in ("walk", "event", "tail", "peel")}
        kernels["launches"] = {k: ws[f"{k}_launches"] for k in ("walk", "event", "tail", "peel")}
        kernels["walks"] = ws["walks"]
        kernels["walk_crossings"] = ws["walk_crossings"]
        kname = f"wave_walk ({args.precision})"
        kms = ws["walk_ms"] / max(ws["walk_launches"], 1)
        abytes = 16.0 * ws["walk_crossings"] / max(ws["walk_launches"], 1)
        if args.traffic_per_walk:
            traffic = args.traffic_per_walk * ws["walks"] / max(ws["walk_launches"], 1)
    else:
        kms = kernel_ms[-1]
        abytes = algorithmic_bytes(counters)
        kname = f"transport_sched ({args.precision})"
    achieved = abytes / (kms / 1e3) / 1e9
    # The timed steps run the wavefront loop as one graph launch per
    # iteration, whose walk times are %globaltimer stamps between the loop's
    # launches.  One more iteration with the host-driven loop times every
    # walk launch with CUDA events on the engine's stream, as a cross-check.
    event_check = None
    if args.schedule == "wave":
        eng.set_wave_loop(False)
        eng.reset_tallies()
        eng.run(np_total, lo, hi, iteration=it, ipeel=args.ipeel)
        wh = eng.wave_stats()
        eng.set_wave_loop(True)
        reduce_ranks(eng)
        event_check = {"walk_ms_per_launch": wh["walk_ms"] / max(wh["walk_launches"], 1),
                       "achieved_gbs": 16.0 * wh["walk_crossings"] / max(wh["walk_launches"], 1)
                       / (wh["walk_ms"] / max(wh["walk_launches"], 1) / 1e3) / 1e9,
                       "how": "host-driven loop, CUDA events around each walk launch, one iteration after the timed steps"}
    # secondary (compute) roofline of the same launches: ~100 FP64 operations
    # per cell crossing (the face quadratics with their square roots and
    # divisions, the compares, the move), against the nominal FP64 vector
    # rate of the part (148 SMs x 64 FMA/clock x 2 at 1965 MHz)
    xings = (abytes / 16.0) if args.schedule == "wave" else counters["crossings"]
    fp64_tflops = 100.0 * xings / (kms / 1e3) / 1e12
    fp64_peak = 148 * 64 * 2 * 1.965e9 / 1e12

    # ---- mixed vs FP64 at equal packet count (same random streams), and the
    # peeled imaging iteration, each measured once
    extra = {}
    if rank == 0 and not args.no_compare:
        from src3_mpi_cfitsio_b200 import model as mdl
        other = "fp64" if args.precision == "mixed" else "mixed"
        itc = it + 1
        base = mdl.tdust_from_tdave(m, td)
        res = {}
        for prec in (args.precision, other):
            eng.set_precision(prec)
            m.grid["tdust"] = base.copy()
            eng.upload_grid()
            eng.tdave = td.copy()
            eng.reset_tallies()
            eng.run(P, iteration=itc, ipeel=0)
            k0 = eng.kernel_ms()
            t0_ = eng.download(images=False)
            tdp, _, _ = eng.update_temperature(P, itc)
            m.grid["tdust"] = base.copy()
            eng.upload_grid()
            eng.reset_tallies()
            eng.run(args.peel_packets, iteration=itc, ipeel=1)
            k1 = eng.kernel_ms()
            t1_ = eng.download(images=True)
            res[prec] = (k0, k1, t0_, t1_, tdp)
        # the plain FP64 GPU path: one thread per packet start to finish
        # (transport_fp64), on a bounded sample of the same iteration
        eng.set_precision("fp64")
        eng.set_schedule("packet")
        m.grid["tdust"] = base.copy()
        eng.upload_grid()
        eng.reset_tallies()
        n_plain = min(P, args.plain_packets)
        eng.run(P, 1, n_plain, iteration=itc, ipeel=0)
        plain_pps = n_plain / (eng.kernel_ms() / 1e3)
        eng.set_schedule(args.schedule)
        eng.set_precision(args.precision)
        a64 = res["fp64"]
        amx = res["mixed"]
        tmask = (a64[4] > 1.0 / 11605.0) & (amx[4] > 1.0 / 11605.0)
        terr = np.abs(amx[4][tmask] / a64[4][tmask] - 1.0)
        c64, cmx = a64[2].counters(), amx[2].counters()
        c64p, cmxp = a64[3].counters(), amx[3].counters()
        extra = {
            "fp64_value": P / (a64[0] / 1e3), "mixed_value": P / (amx[0] / 1e3),
            "mixed_over_fp64": a64[0] / amx[0],
            "fp64_plain": {"packets": n_plain, "packets_per_s": plain_pps,
                           "kernel": "transport_fp64 (one thread per packet, FP64)",
                           "mixed_over_fp64_plain": (P / (amx[0] / 1e3)) / plain_pps},
            "peeled_iteration": {"packets": args.peel_packets,
                                 "fp64_packets_per_s": args.peel_packets / (a64[1] / 1e3),
                                 "mixed_packets_per_s": args.peel_packets / (amx[1] / 1e3),
                                 "mixed_over_fp64": a64[1] / amx[1]},
            "mixed_vs_fp64_error": {"sed_l1": _errors(a64[2], amx[2]).get("si"),
                                    "peeled_sed_l1": _errors(a64[3], amx[3]).get("ti"),
                                    "image_i_l1": _errors(a64[3], amx[3]).get("image_m_i"),
                                    "image_q_l1": _errors(a64[3], amx[3]).get("image_m_q"),
                                    "temperature_median_rel": float(np.median(terr)) if terr.size else None,
                                    "temperature_p99_rel": float(np.quantile(terr, 0.99)) if terr.size else None,
                                    "crossings_rel": cmx["crossings"] / c64["crossings"] - 1.0,
                                    "interactions_rel": cmx["interactions"] / c64["interactions"] - 1.0,
                                    "peel_crossings_rel": (cmxp["peel_cross"] / c64p["peel_cross"] - 1.0
                                                           if c64p["peel_cross"] else None),
                                    "geom_fail": {"mixed": cmx["geom_fail"] + cmxp["geom_fail"],
                                                  "fp64": c64["geom_fail"] + c64p["geom_fail"]},
                                    "note": "same packets and random streams; differences are Monte Carlo "
                                            "divergence of histories after FP32 scattering"},
        }
    # ---- gradient time: the path-replay adjoint of the peeled SED and the
    # 3.6/24/70 um images on the same model (mcrt_adjoint), mixed build
    if rank == 0 and args.grad_packets > 0:
        from src3_mpi_cfitsio_b200 import adjoint as madj
        lam, img = madj.sed_image_weights(m)
        eng.adjoint(min(args.grad_packets, 100000), lam, img, iteration=it + 2)   # warm
        eng.synchronize()
        t0g = time.perf_counter()
        g, Lg = eng.adjoint(args.grad_packets, lam, img, iteration=it + 2)
        grad_wall = time.perf_counter() - t0g
        from src3_mpi_cfitsio_b200.engine import model_density
        pgrad = madj.parameter_gradient(m, g, dlog=model_density(m, device=dev)[2])   # analytic disk-law derivatives
        extra["gradient"] = {"packets": args.grad_packets, "seconds": grad_wall,
                             "device_seconds": eng.kernel_ms() / 1e3, "objective": Lg,
                             "outputs": "peeled SED (all bins) + 3.6/24/70 um images, Stokes I",
                             "wrt": "log rho per cell and component (10 x nr x ntheta); disk parameters",
                             "disk_parameters": pgrad, "precision": args.precision}
        eng.reset_tallies()
    if rank == 0 and args.clumpy_packets > 0:
        extra["clumpy_3d"] = bench_clumpy(args, dev)
    if rank == 0:
        extra["setemiss"] = bench_setemiss(args, dev)
        extra["velocity_terms"] = bench_velocity(args, dev)
    if args.batch_models > 0:                  # every rank: the models are sharded over the ranks
        res = bench_batch(args, dev, rank, world, allreduce if dist else None)
        if rank == 0:
            extra["batch"] = res
    out = dict(
        metric=METRIC, value=value, unit=UNIT, n_gpus=world, steps=args.steps, warmup=args.warmup,
        ms_per_step=ms_steps / args.steps, higher_is_better=True, scaling="weak", vs_baseline=None,
        dtype="f64" if args.precision == "fp64" else "f32+f64",
        data="synthetic (seeded model generator; no reference parameter files)",
        config={"workload": "2-D disk+envelope+cavity (nr=100, ntheta=99, nphi=1), one Lucy iteration of "
                            f"{np_total:.0e} packets, diffusion on, peel-off {'on' if args.ipeel else 'off'}",
                "packets_per_gpu": P, "packets_total": np_total, "peel_off": bool(args.ipeel),
                "precision": args.precision, "schedule": args.schedule,
                "l2": "flushed between steps (256 MiB write); working set L2-resident by design",
                "parallelism": f"packet shards x{world}"},
        e2e={"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        roofline={"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                  "frac": achieved / peak, "traffic": traffic,
                  "peak_source": "measured" if not peaks.get("_fallback") else "fallback",
                  "kernel": kname, "kernel_ms_per_launch": kms, "algorithmic_bytes_per_launch": abytes,
                  "timing": "device-driven loop: %globaltimer stamps between the launches of the timed steps",
                  "cuda_event_check": event_check,
                  "note": "cell walk: L2-resident grid, issue-bound; 16 B per crossing is the "
                          "algorithmic HBM-equivalent traffic"},
        roofline_compute={"achieved": fp64_tflops, "peak": fp64_peak, "unit": "TFLOP/s (FP64)",
                          "frac": fp64_tflops / fp64_peak, "peak_source": "nominal",
                          "flops_per_crossing": 100,
                          "note": "neither HBM nor the FP64 pipe bounds the walk: ncu shows instruction issue "
                                  "on ~68 % of cycles at 32 warps/SM, half of each warp's lanes active"},
        kernels_ms_last_step=kernels,
        # kernels of the last timed step (transport launches counted by the
        # engine, plus tfinal_cells / tfinal_mirror / tfinal_stats /
        # tdust_from_tdave), times the timed steps
        gpu_launches=int((counters["launches"] + 4) * args.steps),
        clocks=clk.summary(),
        counters=counters,
        **extra,
    )
    if rank == 0 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(args)      # a pristine model: the state the GPU steps started from
    eng.close()
    return out


def _cpu_step(b, n, it, cores, ipeel):
    """One CPU Lucy step on the oracle: the packet loop over n packets, then
    tfinal on its tallies (timed, not applied: every step sees the same
    temperature).  Returns seconds."""
    from oracle import oracle
    t0 = time.perf_counter()
    tal, _ = oracle.run(b, n, ipeel=ipeel, threads=cores, iteration=it, images=bool(ipeel))
    oracle.tfinal(b, tal["dtauabs"], n, it, b.tdave0)
    return time.perf_counter() - t0


def _cpu_setup():
    """The oracle built for this host (-march=native, FMA contraction still
    off) and the host description."""
    from oracle import oracle
    oracle.use_native()
    oracle.load()
    return {"cpu_model": oracle.cpu_model(), "build": "g++ -O3 -march=native -ffp-contract=off (oracle/Makefile native)"}


def cpu_baseline(args, m=None, sample=None):
    """The oracle (CPU restatement of the reference loop) on all host cores,
    on the state the GPU arm starts from, and on one core."""
    import numpy as np
    from oracle import oracle
    from src3_mpi_cfitsio_b200 import abi
    host = _cpu_setup()
    if m is None:
        m = build_model(args)
    b = abi.Bundle(m)
    b.tdave0 = np.asarray(m.grid["tdust"], dtype=np.float64).copy()
    cores = os.cpu_count() or 1
    n = sample or args.cpu_sample
    _cpu_step(b, min(n, 20000), 1, cores, args.ipeel)                  # warm caches
    dt = _cpu_step(b, n, 2, cores, args.ipeel)
    n1 = max(n // 20, 1000)
    dt1 = _cpu_step(b, n1, 2, 1, args.ipeel)
    # the emission tables (setemiss) of the model's 8 dust species on the
    # same host threads, beside the GPU build in the "setemiss" key
    t0 = time.perf_counter()
    oracle.setemiss(m.tables["nudust"], m.tables["kappad"], m.tables["adust"], m.tables["nlambda"], threads=cores)
    st = time.perf_counter() - t0
    return {"value": n / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{n} packets of one Lucy iteration (packet loop + tfinal) of the same model at the same "
                      f"converged temperature, {cores} host threads",
            "packets_per_s_one_core": n1 / dt1, **host,
            "setemiss_8_species_ms": 1e3 * st}


def run_reference(args, rank, world):
    """The reference arm: the CPU restatement of the reference's packet loop
    (the Fortran + MPI code cannot be built here) on all host cores, each
    step a bounded sample of the same Lucy iteration at the same converged
    temperature as the GPU arm."""
    if rank != 0:
        return None
    import numpy as np
    from src3_mpi_cfitsio_b200 import abi
    host = _cpu_setup()
    m = build_model(args)
    b = abi.Bundle(m)
    b.tdave0 = np.asarray(m.grid["tdust"], dtype=np.float64).copy()
    cores = os.cpu_count() or 1
    n = args.cpu_sample
    for w in range(args.warmup):
        _cpu_step(b, max(n // 10, 1000), w + 1, cores, args.ipeel)
    times = [_cpu_step(b, n, args.warmup + s + 1, cores, args.ipeel) for s in range(args.steps)]
    v = n * args.steps / sum(times)
    return dict(metric=METRIC, value=v, unit=UNIT, n_gpus=world, steps=args.steps, warmup=args.warmup,
                ms_per_step=1e3 * sum(times) / args.steps, higher_is_better=True, scaling="weak",
                vs_baseline=None, dtype="f64", data="synthetic", impl="reference",
                config={"workload": "2-D disk+envelope+cavity (nr=100, ntheta=99, nphi=1), one Lucy iteration "
                                    "(packet loop + tfinal) at the converged temperature, diffusion on",
                        "packets_per_step": n, "peel_off": bool(args.ipeel), "precision": "fp64"},
                cpu_baseline={"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                              "sample": f"{n} packets per step (packet loop + tfinal), {cores} host threads",
                              **host},
                e2e={"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--schedule", default="wave", choices=["wave", "warp", "packet"])
    ap.add_argument("--packets", type=int, default=100_000_000)
    ap.add_argument("--peel-packets", type=int, default=10_000_000)
    ap.add_argument("--ipeel", type=int, default=0)
    ap.add_argument("--cpu-sample", type=int, default=1_000_000,
                    help="packets per CPU step (reference arm) and of the cpu_baseline sample")
    ap.add_argument("--grad-packets", type=int, default=10_000_000,
                    help="packets of the adjoint-gradient timing (0: skip)")
    ap.add_argument("--plain-packets", type=int, default=5_000_000,
                    help="packets of the plain FP64 per-thread comparison run")
    ap.add_argument("--clumpy-packets", type=int, default=10_000_000,
                    help="packets of the 3-D clumpy peeled-iteration sample (0: skip)")
    ap.add_argument("--batch-models", type=int, default=64, help="models of the batched sweep (0: skip)")
    ap.add_argument("--batch-packets", type=int, default=10_000_000, help="packets per model of the batched sweep")
    ap.add_argument("--batch-tune-packets", type=int, default=1_000_000,
                    help="packets per model of each autotuner trial")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-compare", action="store_true")
    # 691.1 B: dram__bytes_read.sum + dram__bytes_write.sum of one wave_walk
    # launch (FP32 walk, record in 16-byte groups) over 2,097,152 walks, from
    # an ncu capture of the 8e6-packet case
    ap.add_argument("--traffic-per-walk", type=float, default=691.1,
                    help="DRAM bytes per walk of the wave_walk kernel from an ncu capture")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        backend = "gloo" if args.impl == "reference" else "nccl"
        tdist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=600))
    out = run_reference(args, rank, world) if args.impl == "reference" else run_ours(args, rank, world)
    if rank == 0 and out is not None:
        print(json.dumps(out))
    if world > 1:
        import torch.distributed as tdist
        tdist.destroy_process_group()


if __name__ == "__main__":
    main()
