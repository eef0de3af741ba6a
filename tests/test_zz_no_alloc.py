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


def _noalloc(eng, nphot, it, tdave):
    lib = eng.lib
    lib.mcrt_update_temperature_noalloc.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_double),
                                                    C.POINTER(C.c_int32), C.POINTER(C.c_double)]
    lib.mcrt_update_temperature_noalloc.restype = C.c_int
    td = np.ascontiguousarray(tdave, dtype=np.float64).copy()
    conv = C.c_int32(0)
    sig = np.zeros(3)
    rc = lib.mcrt_update_temperature_noalloc(eng.ctx, nphot, it, td.ctypes.data_as(C.POINTER(C.c_double)),
                                             C.byref(conv), sig.ctypes.data_as(C.POINTER(C.c_double)))
    assert rc == 0, lib.mcrt_last_error(eng.ctx)
    return td, sig


def test_noalloc_matches_allocating_entry_point_twice():
    """Two Lucy iterations; after each packet run both entry points update
    the temperature from the same device tallies and must agree."""
    from src3_mpi_cfitsio_b200.engine import Engine
    m = model.warm(model.small_2d())
    n = 20000
    eng = Engine(m)
    tdave = m.grid["tdust"].copy()
    for it in (1, 2):
        eng.reset_tallies()
        eng.run(n, iteration=it, ipeel=0)
        td_b, sig_b = _noalloc(eng, n, it, tdave)
        eng.tdave = tdave
        td_a, _, sig_a = eng.update_temperature(n, it)
        assert np.isfinite(td_b).all() and (td_b > 0).all()
        assert np.allclose(td_b, td_a, rtol=1e-12, atol=0), np.abs(td_b - td_a).max()
        assert np.allclose(sig_b, sig_a, rtol=1e-9, equal_nan=True)
        tdave = td_a
    eng.close()


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
