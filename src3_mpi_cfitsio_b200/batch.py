"""Many models per launch (C ABI ``mcrt_batch_*``; no reference counterpart).

The reference runs one model per MPI job: ``newtts.f90`` calls ``disk`` once
per Lucy iteration for its single grid.  A parameter sweep of that code is
many such jobs.  Here the temperature iterations of a whole sweep share the
GPU: ``Batch.run_iteration`` runs one iteration of every model as one CUDA
graph launch (tally resets, packet loops, diffusion-heating finalisation)
with one of two schedules: "persistent" (one launch whose warps take
(model, packet chunk) items) or "wave" (each model's wavefront loop driven
on the device by a graph WHILE node, the models in parallel branches).
``Batch.tune`` is the autotuner: the schedule, then its knobs (items per
warp, event batch, blocks per SM; or in-flight packet slots per model).  Each model keeps its
own ``Engine`` (context), so the temperature update and the final peel-off
iteration stay per model.

``batch_lucy_iterations`` is the Lucy loop of newtts.f90:225-256 for every
model of a batch at once.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .engine import Engine, MCRTError, load_library

SCHEDULES = {"persistent": 0, "wave": 1}


class Batch:
    """One launch per iteration over the models of `engines` (one device,
    one precision, grids and tables uploaded).  The engines must outlive the
    batch."""

    def __init__(self, engines):
        self.lib = load_library()
        self.engines = list(engines)
        if not self.engines:
            raise ValueError("empty batch")
        arr = (C.c_void_p * len(self.engines))(*[e.ctx for e in self.engines])
        h = C.c_void_p()
        rc = self.lib.mcrt_batch_create(arr, len(self.engines), C.byref(h))
        self.h = h if h.value else None
        self._check(rc)
        self.tuning = None

    def _check(self, rc):
        if rc != 0:
            msg = self.lib.mcrt_batch_last_error(self.h).decode() if self.h else ""
            raise MCRTError(f"mcrt batch call failed (code {rc}): {msg}")

    def close(self):
        if getattr(self, "h", None):
            self.lib.mcrt_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_schedule(self, schedule: str = "persistent", wave_slots: int = 1 << 18):
        """"persistent": one launch over (model, chunk) items; "wave": every
        model's wavefront loop on the device, models in parallel graph
        branches, `wave_slots` in-flight packets per model."""
        self._check(self.lib.mcrt_batch_set_schedule(self.h, SCHEDULES[schedule], int(wave_slots)))

    def set_tuning(self, blocks_per_sm: int = 0, event_batch: int = 16, items_per_warp: int = 4):
        """Knobs of the persistent schedule."""
        self._check(self.lib.mcrt_batch_set_tuning(self.h, blocks_per_sm, event_batch, items_per_warp))

    def tune(self, sample_packets: int) -> dict:
        """Autotune on `sample_packets` per model (overwrites the tallies);
        returns the chosen schedule and knobs."""
        ch = (C.c_int32 * 5)()
        self._check(self.lib.mcrt_batch_tune(self.h, int(sample_packets), ch))
        self.tuning = dict(schedule={v: k for k, v in SCHEDULES.items()}[int(ch[0])], blocks_per_sm=int(ch[1]),
                           event_batch=int(ch[2]), items_per_warp=int(ch[3]), wave_slots=int(ch[4]))
        return self.tuning

    def run_iteration(self, np_per_model, iteration: int = 1, seeds=(12345678, 87654321), generator: int = 1):
        """One iteration of every model (tallies reset first), no peel-offs."""
        n = len(self.engines)
        npm = np.broadcast_to(np.asarray(np_per_model, dtype=np.int64), (n,)).copy()
        self._np = npm
        self._check(self.lib.mcrt_batch_run_iteration(self.h, npm.ctypes.data_as(C.POINTER(C.c_int64)), iteration,
                                                      seeds[0], seeds[1], generator))

    def kernel_ms(self) -> float:
        """Device time of the last iteration's graph launch [ms]."""
        v = C.c_double()
        self._check(self.lib.mcrt_batch_last_ms(self.h, C.byref(v)))
        return v.value


def batch_lucy_iterations(models, np_per_model, n_iter: int, precision: str = "mixed", device: int = 0,
                          tune_packets: int = 0):
    """Lucy iterations (newtts.f90:225-256, no peel-off) of every model, one
    batched launch per iteration; returns (engines, per-iteration device ms).
    The convergence test of each model is evaluated (``Engine.sig``) but the
    loop runs `n_iter` iterations for all, as a sweep with a fixed count."""
    engines = [Engine(m, device=device, precision=precision) for m in models]
    b = Batch(engines)
    if tune_packets:
        b.tune(tune_packets)
    npm = np.broadcast_to(np.asarray(np_per_model, dtype=np.int64), (len(engines),))
    ms = []
    for it in range(1, n_iter + 1):
        b.run_iteration(npm, iteration=it)
        ms.append(b.kernel_ms())
        for e, n in zip(engines, npm):
            e.update_temperature(int(n), it)
    b.close()
    return engines, ms
