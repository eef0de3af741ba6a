"""The allocation-free temperature update against the ordinary one.

mcrt_update_temperature_noalloc exists for drivers that cannot allocate
device memory between Lucy iterations; it must give the same dust
temperatures as mcrt_update_temperature, call after call (its scratch array
persists between calls).  This file sorts last so that a run stopping at the
first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from src3_mpi_cfitsio_b200 import model

pytestmark = pytest.mark.gpu


def _noalloc(eng, nphot, it, tdave, converge=0):
    lib = eng.lib
    lib.mcrt_update_temperature_noalloc.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_double),
                                                    C.POINTER(C.c_int32), C.POINTER(C.c_double)]
    lib.mcrt_update_temperature_noalloc.restype = C.c_int
    td = np.ascontiguousarray(tdave, dtype=np.float64).copy()
    conv = C.c_int32(converge)
    sig = np.zeros(3)
    rc = lib.mcrt_update_temperature_noalloc(eng.ctx, nphot, it, td.ctypes.data_as(C.POINTER(C.c_double)),
                                             C.byref(conv), sig.ctypes.data_as(C.POINTER(C.c_double)))
    assert rc == 0, lib.mcrt_last_error(eng.ctx)
    return td, bool(conv.value), sig


def test_noalloc_matches_allocating_entry_point_twice():
    """Three Lucy iterations on a model with diffusion cells.  Two engines
    each run one half of the packets and both take the sum of the two
    halves' tallies, so they hold the same device state bit for bit (the
    sharded reduction of a multi-GPU run); one then updates the temperature
    with the allocating entry point, the other with the no-alloc one, and
    the temperatures, the convergence statistics and the convergence flag
    must agree call after call (the no-alloc scratch keeps the previous
    call's contents)."""
    from src3_mpi_cfitsio_b200 import dist
    from src3_mpi_cfitsio_b200.engine import Engine
    m = model.with_diffusion(model.warm(model.small_2d()))
    assert (m.grid["diffus"] > 0).any()
    n = 20000
    ea, eb = Engine(m), Engine(m)
    ta = tb = m.grid["tdust"].copy()
    for it in (1, 2, 3):
        for r, e in enumerate((ea, eb)):
            lo, hi = dist.shard_range(n, r, 2)
            e.reset_tallies()
            e.run(n, lo, hi, iteration=it, ipeel=0)
        total = ea.download(images=False).add_(eb.download(images=False))
        for e in (ea, eb):
            e.reset_tallies()
            e.accumulate(total)
            e.refresh_diffusion()
        ea.tdave = ta
        ta, conv_a, sig_a = ea.update_temperature(n, it)
        tb, conv_b, sig_b = _noalloc(eb, n, it, tb)
        assert np.isfinite(tb).all() and (tb > 0).all()
        assert np.allclose(tb, ta, rtol=1e-12, atol=0), np.abs(tb - ta).max()
        assert np.allclose(sig_b, sig_a, rtol=1e-9, equal_nan=True)
        assert conv_a == conv_b
    ea.close()
    eb.close()


def test_noalloc_rejects_models_beyond_its_scratch():
    """A grid above the fixed scratch size is refused with an error code."""
    from src3_mpi_cfitsio_b200.engine import Engine
    m = model.reference_2d(nrg=101, ntg=199, npg=33, nfreq=4, npeel=1, nxhst=3)   # 663,267 cells
    eng = Engine(m)
    lib = eng.lib
    lib.mcrt_update_temperature_noalloc.restype = C.c_int
    td = m.grid["tdust"].copy()
    conv = C.c_int32(0)
    rc = lib.mcrt_update_temperature_noalloc(eng.ctx, 1000, 1, td.ctypes.data_as(C.POINTER(C.c_double)),
                                             C.byref(conv), None)
    assert rc != 0
    assert b"scratch" in lib.mcrt_last_error(eng.ctx)
    eng.close()
