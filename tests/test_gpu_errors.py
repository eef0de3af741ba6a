"""Error paths of the C ABI, made on the host or by a watchdog setting,
never by a device fault: a bad grid is refused at upload, packets given up
by the walk's crossing limit make the run report MCRT_ERR_GEOM, the wave
loop's limit makes it report MCRT_ERR_TIMEOUT, and after each the context
runs the next iteration normally."""
import copy

import numpy as np
import pytest

from src3_mpi_cfitsio_b200 import model

pytestmark = pytest.mark.gpu

ERR_ARG, ERR_UNSUPPORTED, ERR_GEOM, ERR_TIMEOUT = 1, 3, 4, 5


def _engine(m, precision="fp64"):
    from src3_mpi_cfitsio_b200.engine import Engine
    return Engine(m, precision=precision)


def _normal_run(eng, n=4000):
    eng.reset_tallies()
    eng.run(n, ipeel=0)
    c = eng.download(images=False).counters()
    assert c["packets"] == n and c["geom_fail"] == 0


def test_upload_refuses_a_nan_density_and_the_context_stays_usable():
    from src3_mpi_cfitsio_b200.engine import MCRTError
    m = model.warm(model.small_2d())
    eng = _engine(m)
    bad = copy.deepcopy(m)
    d = bad.grid["densarr"].copy()
    d[int(np.flatnonzero(d > 0)[10])] = np.nan
    bad.grid["densarr"] = d
    eng.model = bad
    with pytest.raises(MCRTError) as e:
        eng.upload_grid()
    assert e.value.code == ERR_ARG and "densarr" in str(e.value)
    eng.model = m
    eng.upload_grid()
    _normal_run(eng)
    eng.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_walk_limit_reports_lost_packets(precision):
    """A walk limit of 3 crossings gives up the walks (a packet leaving the
    star crosses more walls than that): their packets are dropped and
    counted, the run returns MCRT_ERR_GEOM with the count, every packet is
    accounted for, and with the default limits the next run is clean."""
    from src3_mpi_cfitsio_b200.engine import MCRTError
    m = model.warm(model.small_2d())
    eng = _engine(m, precision)
    n = 4000
    eng.set_limits(walk_crossings=3)
    eng.reset_tallies()
    with pytest.raises(MCRTError) as e:
        eng.run(n, ipeel=1)
    assert e.value.code == ERR_GEOM and "geometry" in str(e.value)
    c = eng.download(images=False).counters()
    assert c["packets"] == n and c["geom_fail"] > 0
    assert f"{c['geom_fail']} of {n} packets" in str(e.value)
    assert c["exited"] + c["geom_fail"] + c["killed"] == n
    eng.set_limits()
    _normal_run(eng)
    eng.close()


def test_wave_limit_times_out_and_the_next_run_is_whole():
    """Two waves cannot finish 20000 packets in a 1024-slot pool: the run
    stops with MCRT_ERR_TIMEOUT, abandoning the packets in flight; the next
    run of the same context starts a fresh pool and finishes every packet."""
    from src3_mpi_cfitsio_b200.engine import MCRTError
    m = model.warm(model.small_2d())
    eng = _engine(m, "mixed")
    eng.set_schedule("wave")
    eng.set_wave_pool(1024, 0, 0)
    eng.set_limits(waves=2)
    eng.reset_tallies()
    with pytest.raises(MCRTError) as e:
        eng.run(20000, ipeel=0)
    assert e.value.code == ERR_TIMEOUT and "waves" in str(e.value)
    assert eng.download(images=False).counters()["packets"] < 20000
    eng.set_limits()
    _normal_run(eng, 20000)
    eng.close()


def test_small_grains_without_draine_spectra_are_refused():
    """A grid with small-grain components but no Draine spectra uploads, and
    the run refuses it with MCRT_ERR_UNSUPPORTED before any launch; a Draine
    row beyond the table (imean) is MCRT_ERR_ARG; with the spectra the run
    goes through."""
    from src3_mpi_cfitsio_b200.engine import MCRTError
    m = model.with_small_grains(model.warm(model.small_2d()))
    tables = dict(m.tables)
    bare = copy.deepcopy(m)
    for k in ("draine", "nemit", "ndraine"):
        bare.tables.pop(k)
    eng = _engine(bare)
    with pytest.raises(MCRTError) as e:
        eng.run(1000, ipeel=0)
    assert e.value.code == ERR_UNSUPPORTED
    eng.close()
    over = copy.deepcopy(m)
    c = over.config
    over.grid["imean"] = np.full(c["nrg"] * c["ntg"] * c["npg"], tables["nemit"] + 1, np.int32)
    eng = _engine(over)
    with pytest.raises(MCRTError) as e:
        eng.run(1000, ipeel=0)
    assert e.value.code == ERR_ARG
    eng.close()
    eng = _engine(m)
    _normal_run(eng)
    eng.close()
