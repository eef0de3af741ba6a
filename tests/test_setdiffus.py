"""setdiffus (setdiffus_5.f90:1-132) and gridset's temperature reset
(gridset_5_model13new.f90:1842-1866): the oracle's C restatement against the
model generator's (CPU), and the device entry point mcrt_setdiffus against
the oracle (GPU).  Flags are integers and the temperatures are copies, so
every comparison is exact."""
import numpy as np
import pytest

from src3_mpi_cfitsio_b200 import abi, model


def _cases():
    """(name, model, tdave, iteration): the 2-D benchmark grid at the
    power-law stand-in temperature, at a colder field and at a uniform 30 K
    (the first iteration's 50 K floor decides there), the reduced grid, and a 3-D clumpy
    grid (phi slices copied from slice 1)."""
    out = []
    ref = model.warm(model.reference_2d())
    out += [("ref_warm", ref, ref.grid["tdust"].copy(), it) for it in (1, 2)]
    cold = model.warm(model.reference_2d(), t1au_k=120.0, q=0.6)
    out += [("ref_cold", cold, cold.grid["tdust"].copy(), it) for it in (1, 3)]
    floor = model.warm(model.reference_2d(), t1au_k=30.0, q=0.0)
    out.append(("ref_30K", floor, floor.grid["tdust"].copy(), 1))
    small = model.warm(model.small_2d())
    out.append(("small", small, small.grid["tdust"].copy(), 2))
    cl = model.warm(model.clumpy_3d(nrg=41, ntg=41, npg=17, nfreq=20, npeel=4, nxhst=31, rim_walls=8))
    out.append(("clumpy", cl, cl.grid["tdust"].copy(), 2))
    return out


CASES = _cases()


def _rmaxd(m):
    return m.w.rmaxd_au * m.config["autors"]


@pytest.mark.parametrize("case", CASES, ids=[f"{c[0]}-it{c[3]}" for c in CASES])
def test_oracle_setdiffus_matches_the_generator(case, oracle_mod):
    name, m, td, it = case
    d, dd, tdu = oracle_mod.setdiffus(abi.Bundle(m), it, m.w.massd, _rmaxd(m), td)
    g = model.setdiffus(model.Model(m.w), td, it)
    assert np.array_equal(d, g.grid["diffus"])
    assert np.array_equal(dd, g.grid["diffdir"])
    assert np.array_equal(tdu, g.grid["tdust"])
    assert d.sum() > 0, "the case has no diffusion cells"
    w = m.w
    D = d.reshape((w.nrg, w.ntg, w.npg), order="F")
    DD = dd.reshape((w.nrg, w.ntg, w.npg), order="F")
    # upper hemisphere -2, lower +2, the phi slices equal
    up = D[:, : (w.ntg - 1) // 2, :] > 0
    assert (DD[:, : (w.ntg - 1) // 2, :][up] == -2).all()
    lo = D[:, (w.ntg + 1) // 2 - 1:, :] > 0
    assert (DD[:, (w.ntg + 1) // 2 - 1:, :][lo] == 2).all()
    if w.npg > 2:
        assert (D[:, :, 1:w.npg - 1] == D[:, :, :1]).all()


def test_oracle_setdiffus_without_a_disk_flags_nothing(oracle_mod):
    m = model.warm(model.reference_2d())
    td = m.grid["tdust"].copy()
    d, dd, tdu = oracle_mod.setdiffus(abi.Bundle(m), 2, 0.0, _rmaxd(m), td)
    assert d.sum() == 0 and dd.sum() == 0
    empty = m.dens4().sum(axis=-1).ravel(order="F") == 0
    assert np.array_equal(tdu[~empty], td[~empty])
    assert (tdu[empty] == 0.1 / 11605.0).all()


def test_the_region_follows_the_temperature(oracle_mod):
    """The Rosseland mean depends on the temperature, so the region that
    setdiffus flags changes with the field it is given."""
    m = model.warm(model.reference_2d())
    warm = m.grid["tdust"].copy()
    cool = model.warm(model.reference_2d(), t1au_k=120.0, q=0.6).grid["tdust"].copy()
    nw = oracle_mod.setdiffus(abi.Bundle(m), 3, m.w.massd, _rmaxd(m), warm)[0].sum()
    nc = oracle_mod.setdiffus(abi.Bundle(m), 3, m.w.massd, _rmaxd(m), cool)[0].sum()
    assert nw != nc


def test_the_first_iteration_floors_the_temperature_at_50K(oracle_mod):
    """Below 50 K (a uniform 30 K disk) the first iteration's floor
    (setdiffus_5.f90:84) makes the inner disk thick enough to diffuse; later
    iterations use the field as it is."""
    m = model.warm(model.reference_2d())
    td = model.warm(model.reference_2d(), t1au_k=30.0, q=0.0).grid["tdust"].copy()
    n1 = oracle_mod.setdiffus(abi.Bundle(m), 1, m.w.massd, _rmaxd(m), td)[0].sum()
    n3 = oracle_mod.setdiffus(abi.Bundle(m), 3, m.w.massd, _rmaxd(m), td)[0].sum()
    assert n1 > 0 and n3 == 0


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=[f"{c[0]}-it{c[3]}" for c in CASES])
def test_device_setdiffus_matches_the_oracle(case, oracle_mod):
    from src3_mpi_cfitsio_b200.engine import Engine
    name, m, td, it = case
    d, dd, tdu = oracle_mod.setdiffus(abi.Bundle(m), it, m.w.massd, _rmaxd(m), td)
    eng = Engine(m, precision="fp64")
    gd, gdd, cnt = eng.setdiffus(it, td)
    eng.close()
    assert np.array_equal(gd, d)
    assert np.array_equal(gdd, dd)
    w = m.w
    assert cnt == int(d.reshape((w.nrg, w.ntg, w.npg), order="F")[:-1, :-1, :max(w.npg - 1, 1)].sum())


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_runs_after_device_setdiffus_equal_runs_on_the_generated_region(precision):
    """An engine given the model without a diffusion region, then
    mcrt_setdiffus, runs the same packets as one given the generator's
    region at upload: the cell flags and start temperatures are the same.
    Packets that reach a diffusion cell depend on the order in which the
    lanes heat the surface, so those are compared by count only; every
    other packet must have the same history bit for bit."""
    from src3_mpi_cfitsio_b200.engine import Engine
    base = model.warm(model.small_2d())
    td = base.grid["tdust"].copy()
    ref = model.setdiffus(model.warm(model.small_2d()), td, 2)
    assert ref.grid["diffus"].sum() > 0
    n = 20000
    logs = []
    for m, dev in ((ref, False), (base, True)):
        eng = Engine(m, precision=precision)
        if dev:
            eng.setdiffus(2, td)
        eng.enable_packet_log(n)
        eng.reset_tallies()
        eng.run(n, ipeel=0)
        logs.append(abi.packet_log_to_numpy(eng.packet_log(n)))
        eng.close()
    a, b = logs
    nodiff = (a["pad"] == 0) & (b["pad"] == 0)
    assert nodiff.mean() > 0.5
    assert (a["pad"] != 0).sum() == (b["pad"] != 0).sum()
    for k in a:
        assert np.array_equal(a[k][nodiff], b[k][nodiff]), k


@pytest.mark.gpu
def test_setdiffus_without_outputs_feeds_the_convergence_statistics(oracle_mod):
    """mcrt_setdiffus with no output arrays returns without waiting; the
    flags reach tfinal's convergence statistics (which leave diffusion cells
    out) through the temperature update.  Same tallies, same result as the
    call that returns the flags, and as an engine given the region at
    upload."""
    from src3_mpi_cfitsio_b200.engine import Engine
    base = model.warm(model.small_2d())
    td = base.grid["tdust"].copy()
    ref = model.setdiffus(model.warm(model.small_2d()), td, 2)
    tal, _ = oracle_mod.run(abi.Bundle(ref), 20000, ipeel=0, threads=8, images=False)
    res = []
    for m, outputs in ((base, True), (base, False), (ref, None)):
        eng = Engine(m, precision="fp64")
        if outputs is not None:
            eng.setdiffus(2, td, outputs=outputs)
        eng.reset_tallies()
        eng.accumulate(tal)
        eng.tdave = td.copy()
        t, conv, sig = eng.update_temperature(20000, 2)
        res.append((t, sig))
        eng.close()
    assert np.isfinite(res[0][1]).all()
    for t, sig in res[1:]:
        assert np.array_equal(t, res[0][0])
        assert np.array_equal(sig, res[0][1])
