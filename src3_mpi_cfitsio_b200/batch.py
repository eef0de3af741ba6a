"""Many models per launch (C ABI ``mcrt_batch_*``; no reference counterpart).

The reference runs one model per MPI job: ``newtts.f90`` calls ``disk`` once
per Lucy iteration for its single grid.  A parameter sweep of that code is
many such jobs.  Here the temperature iterations of a whole sweep share the
GPU: ``Batch.run_iteration`` runs one iteration of every model in one
persistent launch (work items = (model, packet chunk)), captured in a CUDA
graph together with the tally resets and the diffusion-heating
finalisation; ``Batch.tune`` is the autotuner over blocks per SM, the warp
schedule's event batch and the work items per warp.  Each model keeps its
own ``Engine`` (context), so the temperature update and the final peel-off
iteration stay per model.

``batch_lucy_iterations`` is the Lucy loop of newtts.f90:225-256 for every
model of a batch at once.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .engine import Engine, MCRTError, load_library


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

    def set_tuning(self, blocks_per_sm: int = 0, event_batch: int = 16, items_per_warp: int = 4):
        self._check(self.lib.mcrt_batch_set_tuning(self.h, blocks_per_sm, event_batch, items_per_warp))
        self.tuning = (blocks_per_sm, event_batch, items_per_warp)

    def tune(self, sample_packets: int) -> tuple:
        """Autotune on `sample_packets` per model (overwrites the tallies);
        returns (blocks_per_sm, event_batch, items_per_warp)."""
        ch = (C.c_int32 * 3)()
        self._check(self.lib.mcrt_batch_tune(self.h, int(sample_packets), ch))
        self.tuning = tuple(int(x) for x in ch)
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
