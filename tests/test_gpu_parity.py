"""FP64 engine (CUDA, through the C ABI) against the CPU oracle.

Event-for-event: the same packets draw the same random numbers, take the
same scatter/absorb decisions and end in the same state; the FP64 kernel is
built without FMA contraction, so packets can only part company through a
last-place difference of a transcendental function flipping a comparison.
Tallies: integer tallies agree up to such packets; FP64 sums agree to
1e-9 relative (atomic order); the REAL outputs to float rounding.
"""
import numpy as np
import pytest

from src3_mpi_cfitsio_b200 import abi, model

pytestmark = pytest.mark.gpu


def _engine(m, precision="fp64"):
    from src3_mpi_cfitsio_b200.engine import Engine
    return Engine(m, precision=precision)


def _same_packets(g, o):
    same = ((g["ndraws"] == o["ndraws"]) & (g["nscat"] == o["nscat"]) & (g["nabs"] == o["nabs"]) &
            (g["status"] == o["status"]) & (g["ncross"] == o["ncross"]) & (g["nstar"] == o["nstar"]))
    close = np.isclose(g["nub"], o["nub"], rtol=1e-9, atol=0) & np.isclose(g["sip"], o["sip"], rtol=1e-9, atol=1e-12)
    return same, same & close


@pytest.fixture(scope="module")
def warm_small():
    return model.warm(model.small_2d())


@pytest.mark.parametrize("ipeel", [0, 1])
def test_fp64_event_for_event(warm_small, oracle_mod, ipeel):
    n = 3000 if ipeel else 20000
    eng = _engine(warm_small)
    eng.enable_packet_log(n)
    eng.reset_tallies()
    eng.run(n, ipeel=ipeel)
    g = abi.packet_log_to_numpy(eng.packet_log(n))
    tg = eng.download()
    to, lo = oracle_mod.run(abi.Bundle(warm_small), n, ipeel=ipeel, nlog=n)
    o = abi.packet_log_to_numpy(lo)
    assert (g["iphot"] == np.arange(1, n + 1)).all()
    same, exact = _same_packets(g, o)
    assert same.mean() >= 0.995, same.mean()
    assert exact.mean() >= 0.995, exact.mean()
    assert (g["nscat"] + g["nabs"]).sum() > n // 5      # the model interacts
    # integer tallies: identical up to the few packets that parted company
    for k in ("nabs", "dbig", "killed"):
        assert abs(int(tg[k].sum()) - int(to[k].sum())) <= max(2, int(0.01 * to[k].sum())), k
    # FP64 cell tally
    da, db = tg["dtauabs"], to["dtauabs"]
    assert np.allclose(da.sum(), db.sum(), rtol=2e-3)
    cg, co = tg.counters(), to.counters()
    assert cg["packets"] == co["packets"] == n
    assert abs(cg["crossings"] - co["crossings"]) <= 0.01 * co["crossings"]
    # SEDs (REAL): total flux per frequency bin
    for k in ("si", "nums", "sq"):
        a = tg.shaped(k)[..., 0].sum(axis=(1, 2, 3))
        b = to.shaped(k)[..., 0].sum(axis=(1, 2, 3))
        assert np.allclose(a, b, rtol=2e-2, atol=2e-3 * np.abs(b).max() + 1e-6), k
    if ipeel:
        for k in ("ti", "tq", "numt"):
            a, b = tg[k].astype(np.float64), to[k].astype(np.float64)
            assert np.allclose(a.sum(), b.sum(), rtol=1e-2), k
        ia, ib = tg["image_m_i"].astype(np.float64), to["image_m_i"].astype(np.float64)
        assert np.allclose(ia.sum(), ib.sum(), rtol=1e-2)
        assert np.abs(ia - ib).max() <= 2e-2 * ib.max()
    eng.close()


@pytest.mark.parametrize("iteration,ipeel,imean", [(1, 0, False), (2, 0, False), (2, 1, True)])
def test_small_grain_packets_event_for_event(warm_small, oracle_mod, iteration, ipeel, imean):
    """Small grains (ids 6-8) with a small-grain-only cavity: packets that
    small grains absorb there re-emit from the Draine spectra
    (rep_draine_new.f90, emit_sg.f90).  Engine and oracle agree packet by
    packet in the first iteration (Draine row 2), a later one (row 1) and
    with a per-cell row (imean); the small-grain absorptions agree."""
    import copy
    m = model.with_small_grains(copy.deepcopy(warm_small))
    if imean:
        c = m.config
        rng = np.random.default_rng(7)
        m.grid["imean"] = rng.integers(1, 19, c["nrg"] * c["ntg"] * c["npg"]).astype(np.int32)
    n = 3000 if ipeel else 20000
    eng = _engine(m)
    eng.enable_packet_log(n)
    eng.reset_tallies()
    eng.run(n, ipeel=ipeel, iteration=iteration)
    g = abi.packet_log_to_numpy(eng.packet_log(n))
    tg = eng.download()
    eng.close()
    to, lo = oracle_mod.run(abi.Bundle(m), n, ipeel=ipeel, nlog=n, iteration=iteration)
    o = abi.packet_log_to_numpy(lo)
    same, exact = _same_packets(g, o)
    assert same.mean() >= 0.995, same.mean()
    assert tg["dsg"].sum() > 0
    assert abs(int(tg["dsg"].sum()) - int(to["dsg"].sum())) <= max(2, int(0.01 * to["dsg"].sum()))
    for k in ("si", "nums"):
        a = tg.shaped(k)[..., 0].sum(axis=(1, 2, 3))
        b = to.shaped(k)[..., 0].sum(axis=(1, 2, 3))
        assert np.allclose(a, b, rtol=2e-2, atol=2e-3 * np.abs(b).max() + 1e-6), k


def test_exact_subset_bitwise(warm_small, oracle_mod):
    """Packets that never touch a transcendental tie end bit-identical in
    their integer state and within 1e-12 in their FP64 state."""
    n = 2000
    eng = _engine(warm_small)
    eng.enable_packet_log(n)
    eng.reset_tallies()
    eng.run(n, ipeel=0)
    g = abi.packet_log_to_numpy(eng.packet_log(n))
    _, lo = oracle_mod.run(abi.Bundle(warm_small), n, ipeel=0, nlog=n)
    o = abi.packet_log_to_numpy(lo)
    same, _ = _same_packets(g, o)
    for k in ("xp", "yp", "zp", "cost", "phi", "nub"):
        rel = np.abs(g[k][same] - o[k][same]) / np.maximum(np.abs(o[k][same]), 1e-300)
        assert np.median(rel) < 1e-13 and np.quantile(rel, 0.99) < 1e-9, k
    eng.close()


def test_tfinal_matches_oracle(warm_small, oracle_mod):
    """Device tfinal/dusttemp against the oracle on the same dtauabs."""
    n = 20000
    eng = _engine(warm_small)
    eng.reset_tallies()
    eng.run(n, ipeel=0)
    tg = eng.download(images=False)
    for it in (1, 4):
        eng.tdave = warm_small.grid["tdust"].copy()
        td_g, _, sig_g = eng.update_temperature(n, it)
        td_o, sig_o = oracle_mod.tfinal(abi.Bundle(warm_small), tg["dtauabs"], n, it, warm_small.grid["tdust"])
        assert np.allclose(td_g, td_o, rtol=1e-12, atol=0), np.abs(td_g - td_o).max()
        assert np.allclose(sig_g, sig_o, rtol=1e-9, equal_nan=True)
    eng.close()


def test_tfinal_with_velocity_field_matches_oracle(oracle_mod):
    """tfinal with the envelope's infall field on the benchmark grid (the
    passes of tfinal_5_test1.f90: smoothed temperatures and gradients,
    dusttemp's adiabatic and advective terms), device against oracle on the
    same dtauabs, one pass (iteration 2) and twenty averaged over the last
    ten (iteration 5).  The diffusion flags are cleared so that every cell
    goes through dusttemp."""
    import copy
    m = model.with_velocities(model.reference_2d_converged())
    m.grid["diffus"] = np.zeros_like(m.grid["diffus"])
    m.grid["diffdir"] = np.zeros_like(m.grid["diffdir"])
    rest = copy.deepcopy(m)
    for k in ("vrarr", "vthetarr", "divvarr"):
        del rest.grid[k]
    n = 200000
    eng = _engine(m)
    eng.reset_tallies()
    eng.run(n, ipeel=0)
    tg = eng.download(images=False)
    env = (m.dens4()[..., 2] > 0).ravel(order="F")
    for it in (2, 5):
        eng.tdave = m.grid["tdust"].copy()
        td_g, _, sig_g = eng.update_temperature(n, it)
        td_o, sig_o = oracle_mod.tfinal(abi.Bundle(m), tg["dtauabs"], n, it, m.grid["tdust"])
        assert np.allclose(td_g, td_o, rtol=1e-12, atol=0), np.abs(td_g / td_o - 1).max()
        assert np.allclose(sig_g, sig_o, rtol=1e-9, equal_nan=True)
        td_r, _ = oracle_mod.tfinal(abi.Bundle(rest), tg["dtauabs"], n, it, m.grid["tdust"])
        change = np.abs(td_g / td_r - 1.0)
        assert change[env].max() > 1e-4 and change[~env].max() <= 1e-12
    eng.close()


def test_multi_launch_sharding(warm_small):
    """Packet ranges are independent: two launches over halves of the range
    give the tallies of one launch over all of it (the per-rank split of the
    MPI run, newtts.f90:139)."""
    n = 4000
    eng = _engine(warm_small)
    eng.reset_tallies()
    eng.run(n, ipeel=1)
    a = eng.download()
    eng.reset_tallies()
    eng.run(n, 1, n // 2, ipeel=1)
    eng.run(n, n // 2 + 1, n, ipeel=1)
    b = eng.download()
    for k in ("nabs", "dbig", "killed"):
        assert (a[k] == b[k]).all(), k
    assert np.allclose(a["dtauabs"], b["dtauabs"], rtol=1e-12, atol=1e-300)
    for k in ("si", "ti", "image_m_i"):
        assert np.allclose(a[k], b[k], rtol=1e-5, atol=1e-6 * max(1e-30, np.abs(a[k]).max())), k
    eng.close()


def test_errors_are_reported_not_fatal(warm_small):
    from src3_mpi_cfitsio_b200.engine import MCRTError
    eng = _engine(warm_small)
    with pytest.raises(MCRTError):
        eng.run(100, 50, 200)          # range beyond np
    with pytest.raises(MCRTError):
        eng.run(100, generator=40)     # generator outside 1..32
    eng.run(100)                        # context still usable
    assert eng.download(images=False).counters()["packets"] == 100
    eng.close()


@pytest.fixture(scope="module")
def diffusion_small():
    return model.with_diffusion(model.warm(model.small_2d()))


@pytest.mark.parametrize("schedule", ["warp", "wave"])
def test_diffusion_statistical_and_pre_diffusion_exact(diffusion_small, oracle_mod, schedule):
    """Diffusion (emit_common_2.f90:201-372): packets that never reach a
    diffusion cell stay event-for-event equal; the ones that do depend on
    the order in which diffusion absorptions heat the surface cell, so the
    ensemble is compared within Monte Carlo error."""
    m = diffusion_small
    n = 20000
    eng = _engine(m)
    eng.set_schedule(schedule)
    if schedule == "wave":
        eng.set_wave_pool(2048)
    eng.enable_packet_log(n)
    eng.reset_tallies()
    eng.run(n, ipeel=0)
    g = abi.packet_log_to_numpy(eng.packet_log(n))
    tg = eng.download(images=False)
    to, lo = oracle_mod.run(abi.Bundle(m), n, ipeel=0, nlog=n)
    o = abi.packet_log_to_numpy(lo)
    nodiff = (g["pad"] == 0) & (o["pad"] == 0)
    assert g["pad"].sum() > 20 and o["pad"].sum() > 20       # the diffusion branch runs
    same, exact = _same_packets(g, o)
    assert exact[nodiff].mean() >= 0.995
    # diffusion events: same count up to Monte Carlo noise
    dg, do = g["pad"].sum(), o["pad"].sum()
    assert abs(dg - do) <= 5 * np.sqrt(do) + 5
    assert (g["status"] == 3).sum() == 0
    # SED of the ensemble
    a = tg.shaped("nums")[..., 0].sum(axis=(1, 2, 3))
    b = to.shaped("nums")[..., 0].sum(axis=(1, 2, 3))
    assert np.all(np.abs(a - b) <= 5 * np.sqrt(np.maximum(b, 1)) + 5)
    eng.close()


@pytest.mark.parametrize("batch", [1, 12, 32])
def test_schedules_agree_bitwise(warm_small, batch):
    """The warp-scheduled kernel reorders work across lanes, never within a
    packet: its packet logs equal the per-thread kernel's bit for bit."""
    n = 3000
    logs = []
    for sched in ("packet", "warp"):
        eng = _engine(warm_small)
        eng.set_schedule(sched, batch)
        eng.enable_packet_log(n)
        eng.reset_tallies()
        eng.run(n, ipeel=1)
        logs.append(abi.packet_log_to_numpy(eng.packet_log(n)))
        eng.close()
    a, b = logs
    for k in a:
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("precision,pool,tail", [("fp64", 1 << 21, -1), ("mixed", 2048, -1), ("mixed", 1024, 0)])
def test_device_wave_loop_matches_host_loop(warm_small, precision, pool, tail):
    """The wavefront loop as one graph launch (the device decides on the
    next wave and on the tail launch) runs the same packets as the
    host-driven loop: packet logs bit for bit, counters exactly, tallies up
    to FP64 summation order; a second iteration reuses the captured graph
    with the iteration's random blocks, and the loop's own timings account
    for every wave."""
    n = 20000
    out = []
    for device in (False, True):
        eng = _engine(warm_small, precision=precision)
        eng.set_schedule("wave")
        eng.set_wave_pool(pool, 0, tail)
        eng.set_wave_loop(device)
        eng.enable_packet_log(n)
        logs, tals, stats = [], [], []
        for it in (1, 2):
            eng.reset_tallies()
            eng.run(n, ipeel=0, iteration=it)
            logs.append(abi.packet_log_to_numpy(eng.packet_log(n)))
            tals.append(eng.download(images=False))
            stats.append(eng.wave_stats())
        eng.close()
        out.append((logs, tals, stats))
    (lh, th, sh), (ld, td, sd) = out
    for it in range(2):
        for k in lh[it]:
            assert np.array_equal(lh[it][k], ld[it][k]), (it, k)
        ch, cd = th[it].counters(), td[it].counters()
        for k in ("packets", "crossings", "interactions", "scatters", "killed", "exited", "starhits", "waves"):
            assert ch[k] == cd[k], (it, k)
        assert np.allclose(th[it]["dtauabs"], td[it]["dtauabs"], rtol=1e-10, atol=1e-12 * th[it]["dtauabs"].max())
        assert np.array_equal(th[it]["nabs"], td[it]["nabs"])
        assert sd[it]["walk_launches"] == sh[it]["walk_launches"] == ch["waves"]
        assert sd[it]["walks"] == sh[it]["walks"] and sd[it]["walk_crossings"] == sh[it]["walk_crossings"]
        assert sd[it]["walk_ms"] > 0 and sd[it]["event_ms"] > 0
    assert not np.array_equal(ld[0]["ndraws"], ld[1]["ndraws"])       # the second iteration drew other blocks


@pytest.mark.parametrize("precision,pool,batch,tail", [("fp64", 1 << 21, 8, -1), ("fp64", 96, 1, 0),
                                                       ("fp64", 512, 32, 200), ("mixed", 1 << 21, 8, -1),
                                                       ("mixed", 256, 8, 0)])
def test_wave_schedule_matches_warp_bitwise(warm_small, precision, pool, batch, tail):
    """The wavefront schedule (walk and event kernels over a pool of
    in-flight packets in HBM, then one tail launch for the last packets)
    runs every packet's steps in the same order on the same random stream as
    the warp schedule: packet logs agree bit for bit, counters exactly,
    tallies up to FP64 summation order.  Small pools take many waves and
    drain the peel-off job queue more than once; tail 0 waves to the end."""
    n = 3000
    logs, tals = [], []
    for sched in ("warp", "wave"):
        eng = _engine(warm_small, precision=precision)
        eng.set_schedule(sched, batch if sched == "wave" else 16)
        if sched == "wave":
            eng.set_wave_pool(pool, 2 * pool if pool < 1000 else 0, tail)
        eng.enable_packet_log(n)
        eng.reset_tallies()
        eng.run(n, ipeel=1)
        logs.append(abi.packet_log_to_numpy(eng.packet_log(n)))
        tals.append(eng.download())
        eng.close()
    a, b = logs
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    ca, cb = tals[0].counters(), tals[1].counters()
    assert cb["waves"] > 0 and ca["waves"] == 0
    for k in ("packets", "crossings", "interactions", "scatters", "peels", "peel_cross", "peel_binned",
              "geom_fail", "resets", "killed", "exited", "starhits"):
        assert ca[k] == cb[k], k
    # the waves never overflow the job queue; the tail launch walks the
    # peel-offs of a full queue inline, as the warp kernel does
    if tail == 0:
        assert ca["peel_jobs"] == cb["peel_jobs"]
    else:
        assert cb["peel_jobs"] <= ca["peel_jobs"]
    if tail == 0:
        assert cb["waves"] > n // pool
    for k in ("ti", "tq", "tu", "numt", "image_m_i", "image_m_q", "si", "sq", "nums", "dtauabs"):
        x, y = tals[0][k], tals[1][k]
        assert np.allclose(x, y, rtol=1e-5, atol=1e-6 * max(1e-30, float(np.abs(x).max()))), k
    for k in ("nabs", "dbig", "dsg", "killed"):
        assert np.array_equal(tals[0][k], tals[1][k]), k


def test_wave_schedule_without_peel_offs_and_shards(warm_small):
    """Wavefront runs of packet sub-ranges add up to the full range run with
    the warp schedule (the sharding used across ranks)."""
    n = 4000
    eng = _engine(warm_small)
    eng.set_schedule("warp")
    eng.reset_tallies()
    eng.run(n, ipeel=0)
    a = eng.download()
    eng.close()
    eng = _engine(warm_small)
    eng.set_schedule("wave")
    eng.set_wave_pool(256, 0, 100)
    eng.reset_tallies()
    for lo, hi in ((1, 1234), (1235, 3001), (3002, 4000)):
        eng.run(n, lo, hi, ipeel=0)
    b = eng.download()
    eng.close()
    ca, cb = a.counters(), b.counters()
    for k in ("packets", "crossings", "interactions", "exited", "starhits"):
        assert ca[k] == cb[k], k
    for k in ("si", "nums", "dtauabs"):
        assert np.allclose(a[k], b[k], rtol=1e-5, atol=1e-6 * max(1e-30, float(np.abs(a[k]).max()))), k
    assert np.array_equal(a["nabs"], b["nabs"])


def test_peel_queue_matches_inline_peel_offs(warm_small):
    """Queued peel-offs (peel-off kernel) give the tallies of peel-offs walked
    inline by the packet's own thread, up to FP64 summation order."""
    n = 4000
    tals = []
    for sched in ("packet", "warp"):
        eng = _engine(warm_small)
        eng.set_schedule(sched, 16)
        eng.reset_tallies()
        eng.run(n, ipeel=1)
        tals.append(eng.download())
        eng.close()
    a, b = tals
    ca, cb = a.counters(), b.counters()
    assert cb["peel_jobs"] > 0 and ca["peel_jobs"] == 0
    for k in ("peels", "peel_cross", "peel_binned", "packets", "crossings", "interactions"):
        assert ca[k] == cb[k], k
    assert cb["peel_resets"] == 0
    for k in ("ti", "tq", "tu", "numt", "image_m_i", "image_m_q", "si", "nums"):
        assert np.allclose(a[k], b[k], rtol=1e-5, atol=1e-6 * max(1e-30, float(np.abs(a[k]).max()))), k


def test_mixed_precision_agrees_with_fp64(oracle_mod):
    """The mixed build (FP32 closest-approach walk and FP32 scattering) runs
    the same random streams as the FP64 build, but its walk places faces to
    FP32 precision, so histories part company and the comparison is
    statistical: per-packet crossing and interaction counts agree within
    4 standard errors, no packet is lost, and every ensemble tally agrees
    far inside the Monte Carlo error."""
    m = model.with_diffusion(model.warm(model.small_2d()))
    n = 40000
    out, logs = {}, {}
    for prec in ("fp64", "mixed"):
        eng = _engine(m, precision=prec)
        eng.enable_packet_log(n)
        eng.reset_tallies()
        eng.run(n, ipeel=1)
        out[prec] = eng.download()
        logs[prec] = abi.packet_log_to_numpy(eng.packet_log(n))
        eng.close()
    a, b = out["fp64"], out["mixed"]
    cb = b.counters()
    assert cb["geom_fail"] == 0 and cb["packets"] == n
    for k in ("ncross", "nscat", "nabs"):
        x, y = logs["fp64"][k].astype(np.float64), logs["mixed"][k].astype(np.float64)
        se = np.sqrt((x.var() + y.var()) / n)
        assert abs(x.mean() - y.mean()) <= 4.0 * se + 1e-9, (k, x.mean(), y.mean(), se)
    for k in ("nums", "si", "numt", "ti", "image_m_i"):
        x, y = a[k].astype(np.float64), b[k].astype(np.float64)
        assert abs(y.sum() - x.sum()) <= 0.02 * abs(x.sum()) + 1e-12, k
        assert np.abs(y - x).sum() <= 0.08 * np.abs(x).sum() + 1e-12, k
    assert np.abs(b["dtauabs"] - a["dtauabs"]).sum() <= 0.05 * np.abs(a["dtauabs"]).sum()


def _with_accretion(m, frac=0.3):
    import copy
    a = copy.deepcopy(m)
    a.config["accfrac"] = frac
    return a


def test_accretion_packets_event_for_event(warm_small, oracle_mod):
    """Disk-accretion packets (initpacc_4.f90, newdisktherm_5_fuv.f90:238-287):
    emission point from the Ldint CDF, rantheta and gasdev, emit_common,
    peel-offs of the isotropic emission, then propagate -- packet for packet
    against the oracle on the model without the diffusion treatment (where
    every packet is deterministic), peel-offs on."""
    m = _with_accretion(warm_small)
    n = 2000
    npacc = int(n * 0.3)
    eng = _engine(m)
    eng.enable_packet_log(n)
    eng.reset_tallies()
    eng.run(n, ipeel=1)
    g = abi.packet_log_to_numpy(eng.packet_log(n))
    tg = eng.download()
    to, lo = oracle_mod.run(abi.Bundle(m), n, ipeel=1, nlog=n)
    o = abi.packet_log_to_numpy(lo)
    acc = g["iphot"] < npacc
    assert acc.sum() == npacc - 1
    same, exact = _same_packets(g, o)
    assert exact[acc].mean() >= 0.995 and exact.mean() >= 0.995
    assert (g["status"][acc] != 3).all()
    assert (g["i_orig"][acc & (g["nabs"] == 0)] == 2).all()     # never absorbed: still an accretion photon
    for k in ("nabs", "dbig", "killed"):
        assert abs(int(tg[k].sum()) - int(to[k].sum())) <= max(2, int(0.01 * to[k].sum())), k
    assert tg["nabs"].sum() >= npacc - 1
    for k in ("ti", "numt"):
        assert np.allclose(tg[k].astype(np.float64).sum(), to[k].astype(np.float64).sum(), rtol=1e-2), k
    eng.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_accretion_wave_matches_warp_bitwise(warm_small, precision):
    m = _with_accretion(model.with_diffusion(warm_small))
    n = 3000
    logs = []
    for sched in ("warp", "wave"):
        eng = _engine(m, precision=precision)
        eng.set_schedule(sched)
        if sched == "wave":
            eng.set_wave_pool(256, 0, 64)
        eng.enable_packet_log(n)
        eng.reset_tallies()
        eng.run(n, ipeel=1)
        logs.append(abi.packet_log_to_numpy(eng.packet_log(n)))
        eng.close()
    a, b = logs
    # diffusion emission depends on the order of surface heating: compare
    # the packets that never reached a diffusion cell bit for bit
    nod = (a["pad"] == 0) & (b["pad"] == 0)
    assert nod.sum() > n // 2
    for k in a:
        assert np.array_equal(a[k][nod], b[k][nod]), k
    assert (b["status"] == 0).all()


@pytest.fixture(scope="module")
def mueller_small():
    return model.with_mueller(model.warm(model.small_2d()), s34_frac=0.6)


@pytest.mark.parametrize("ipeel", [0, 1])
def test_tabulated_scattering_event_for_event(mueller_small, oracle_mod, ipeel):
    """stokes6 / stokespeel6 with tabulated matrices (S34 on), engine vs
    oracle packet for packet; peel-offs through the job queue carry the
    table row and wavelength weight."""
    m = mueller_small
    n = 3000
    eng = _engine(m)
    eng.enable_packet_log(n)
    eng.reset_tallies()
    eng.run(n, ipeel=ipeel)
    g = abi.packet_log_to_numpy(eng.packet_log(n))
    tg = eng.download()
    to, lo = oracle_mod.run(abi.Bundle(m), n, ipeel=ipeel, nlog=n)
    o = abi.packet_log_to_numpy(lo)
    same, exact = _same_packets(g, o)
    assert exact.mean() >= 0.995
    both = same & (g["nscat"] > 0)
    assert both.sum() > 100
    assert np.allclose(g["svp"][both], o["svp"][both], rtol=1e-9, atol=1e-12)
    assert np.abs(g["svp"][both]).max() > 1e-3
    if ipeel:
        for k in ("ti", "tq", "tv", "numt", "image_m_i", "image_m_v"):
            a, b = tg[k].astype(np.float64).sum(), to[k].astype(np.float64).sum()
            assert abs(a - b) <= 1e-2 * max(abs(b), 1e-6 * tg["ti"].astype(np.float64).sum()), k
    eng.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_tabulated_scattering_wave_matches_warp_bitwise(mueller_small, precision):
    n = 3000
    logs = []
    for sched in ("warp", "wave"):
        eng = _engine(mueller_small, precision=precision)
        eng.set_schedule(sched)
        if sched == "wave":
            eng.set_wave_pool(512, 0, 100)
        eng.enable_packet_log(n)
        eng.reset_tallies()
        eng.run(n, ipeel=1)
        logs.append(abi.packet_log_to_numpy(eng.packet_log(n)))
        eng.close()
    a, b = logs
    for k in a:
        assert np.array_equal(a[k], b[k]), k


@pytest.fixture(scope="module")
def clumpy_small():
    """The 3-D clumpy workload in miniature: fractal clumps, 3-D walls
    (phi planes), tabulated Mueller matrices with S34."""
    return model.with_mueller(model.warm(model.clumpy_3d(nrg=41, ntg=41, npg=17, nfreq=20, npeel=4,
                                                         nxhst=31, rim_walls=8)), s34_frac=0.3)


def test_clumpy_3d_event_for_event(clumpy_small, oracle_mod):
    m = clumpy_small
    n = 3000
    eng = _engine(m)
    eng.enable_packet_log(n)
    eng.reset_tallies()
    eng.run(n, ipeel=1)
    g = abi.packet_log_to_numpy(eng.packet_log(n))
    tg = eng.download()
    to, lo = oracle_mod.run(abi.Bundle(m), n, ipeel=1, nlog=n)
    o = abi.packet_log_to_numpy(lo)
    same, exact = _same_packets(g, o)
    assert exact.mean() >= 0.99
    cg, co = tg.counters(), to.counters()
    assert cg["geom_fail"] == co["geom_fail"] == 0
    assert abs(cg["crossings"] - co["crossings"]) <= 0.01 * co["crossings"]
    for k in ("ti", "numt", "image_m_i"):
        a, b = tg[k].astype(np.float64).sum(), to[k].astype(np.float64).sum()
        assert abs(a - b) <= 2e-2 * abs(b), k
    eng.close()


def test_clumpy_3d_mixed_wave_loses_no_packets(clumpy_small):
    """Mixed build on the 3-D walls: no geometry failures, ensemble within
    the Monte Carlo error of the FP64 build."""
    n = 20000
    out = {}
    for prec in ("fp64", "mixed"):
        eng = _engine(clumpy_small, precision=prec)
        eng.reset_tallies()
        eng.run(n, ipeel=1)
        out[prec] = eng.download()
        eng.close()
    a, b = out["fp64"], out["mixed"]
    assert b.counters()["geom_fail"] == 0 and b.counters()["packets"] == n
    for k in ("nums", "numt"):
        x, y = a[k].astype(np.float64).sum(), b[k].astype(np.float64).sum()
        assert abs(y - x) <= 0.02 * x + 50, k


def _adjoint_weights(m):
    c = m.config
    lam = np.zeros((c["nfreq"], c["npeel"], c["nap"], 8))
    lam[:, :, :, 0] = np.linspace(0.5, 1.5, c["nfreq"])[:, None, None]
    img = np.linspace(0.2, 1.0, c["npeel"] * c["nxhst"] ** 2 * c["nfreq"])
    return lam.ravel(order="F"), img


@pytest.mark.parametrize("diffusion", [False, True])
def test_adjoint_matches_oracle(warm_small, oracle_mod, diffusion):
    """mcrt_adjoint (forward pass through the wave and peel-off kernels,
    records sorted on the device, replay through the warp schedule) against
    the oracle's sequential path replay on the same packets: the same
    objective and dL/dlog(rho) per (cell, component) up to the order of the
    FP64 sums and the rare packet that parts company."""
    m = model.with_diffusion(warm_small) if diffusion else warm_small
    lam, img = _adjoint_weights(m)
    n = 4000
    eng = _engine(m)
    eng.reset_tallies()
    g_gpu, L_gpu = eng.adjoint(n, lam, img)
    eng.close()
    g_or, L_or = oracle_mod.adjoint(abi.Bundle(m), n, lam, img)
    assert L_gpu > 0
    assert abs(L_gpu - L_or) <= 1e-3 * abs(L_or)
    assert np.abs(g_gpu - g_or).sum() <= 2e-2 * np.abs(g_or).sum()
    ncell = m.config["nrg"] * m.config["ntg"] * m.config["npg"]
    for comp in range(10):
        a = g_gpu.reshape((ncell, 10), order="F")[:, comp].sum()
        b = g_or.reshape((ncell, 10), order="F")[:, comp].sum()
        assert abs(a - b) <= 2e-2 * np.abs(g_or.reshape((ncell, 10), order="F")[:, comp]).sum() + 1e-12, comp


def test_adjoint_control_variate_matches_oracle(warm_small, oracle_mod):
    """mcrt_adjoint with the replay's control variate (pilot replay on
    generator 2, mean future contribution per cell x 5 frequency bins x 4
    direction classes) against the oracle doing the same two steps: the
    pilot's counts and the baseline table follow from the same packets, so
    the gradients agree as closely as the plain replay's do."""
    m = model.with_diffusion(warm_small)
    lam, img = _adjoint_weights(m)
    n, pilot = 4000, 3000
    eng = _engine(m)
    eng.set_adjoint_baseline(nfb=5, ndir=4, pilot_packets=pilot, min_count=4.0)
    g_gpu, L_gpu = eng.adjoint(n, lam, img)
    eng.set_adjoint_baseline(nfb=0)
    g_plain, _ = eng.adjoint(n, lam, img)
    eng.close()
    b = abi.Bundle(m)
    _, _, vs, vc = oracle_mod.adjoint_cv(b, pilot, lam, img, nfb=-5, learn=True, generator=2)
    V = np.where(vc >= 4.0, vs / np.maximum(vc, 1.0), 0.0)
    g_or, L_or, _, _ = oracle_mod.adjoint_cv(b, n, lam, img, vtab=V, nfb=-5)
    assert L_gpu > 0 and abs(L_gpu - L_or) <= 1e-3 * abs(L_or)
    assert np.abs(g_gpu - g_or).sum() <= 2e-2 * np.abs(g_or).sum()
    assert np.abs(g_gpu - g_plain).sum() > 1e-3 * np.abs(g_plain).sum()   # the baseline took effect
    ncell = m.config["nrg"] * m.config["ntg"] * m.config["npg"]
    for comp in range(10):
        a = g_gpu.reshape((ncell, 10), order="F")[:, comp].sum()
        o = g_or.reshape((ncell, 10), order="F")[:, comp]
        assert abs(a - o.sum()) <= 2e-2 * np.abs(o).sum() + 1e-12, comp


def test_adjoint_mixed_precision_and_repeatability(warm_small):
    m = model.with_diffusion(warm_small)
    lam, img = _adjoint_weights(m)
    n = 20000
    out = {}
    for prec in ("fp64", "mixed"):
        eng = _engine(m, precision=prec)
        g1, L1 = eng.adjoint(n, lam, img)
        g2, L2 = eng.adjoint(n, lam, img)
        eng.close()
        # the same paths; only the order of the FP64 atomic sums differs
        assert abs(L1 - L2) <= 1e-12 * abs(L1) and np.allclose(g1, g2, rtol=1e-9, atol=1e-12 * np.abs(g1).max())
        out[prec] = (g1, L1)
    (ga, La), (gb, Lb) = out["fp64"], out["mixed"]
    assert abs(Lb - La) <= 0.01 * La
    ncell = m.config["nrg"] * m.config["ntg"] * m.config["npg"]
    for comp in (2, 3):
        a = ga.reshape((ncell, 10), order="F")[:, comp].sum()
        b = gb.reshape((ncell, 10), order="F")[:, comp].sum()
        assert abs(b - a) <= 0.1 * abs(a), comp


def test_adjoint_chunks_sum_to_one_pass(warm_small):
    """mcrt_adjoint in packet chunks (forward, sort and replay per chunk)
    gives the single pass's gradient and objective: the packets are
    independent with diffusion heating frozen."""
    m = model.with_diffusion(warm_small)
    lam, img = _adjoint_weights(m)
    n = 6000
    eng = _engine(m)
    g1, L1 = eng.adjoint(n, lam, img)
    eng.set_adjoint_chunk(1500)
    g2, L2 = eng.adjoint(n, lam, img)
    eng.set_adjoint_chunk(777)                 # ragged last chunk
    g3, L3 = eng.adjoint(n, lam, img, lo=1001, hi=n)
    eng.set_adjoint_chunk(1 << 23)
    g4, L4 = eng.adjoint(n, lam, img, lo=1001, hi=n)
    eng.close()
    assert abs(L2 - L1) <= 1e-12 * abs(L1) and abs(L4 - L3) <= 1e-12 * abs(L4)
    tol = 1e-9 * np.abs(g1).max()
    assert np.allclose(g1, g2, rtol=1e-9, atol=tol) and np.allclose(g3, g4, rtol=1e-9, atol=tol)
    assert L3 < L1


@pytest.fixture(scope="module")
def isrf_small():
    return model.with_isrf(model.with_diffusion(model.warm(model.small_2d())), 0.3)


@pytest.mark.parametrize("ipeel", [0, 1])
def test_isrf_packets_event_for_event(isrf_small, oracle_mod, ipeel):
    """External-illumination packets (30 % of the iteration) follow the
    oracle packet by packet; diffusion is on, so only packets that reach a
    diffusion cell may part company."""
    m = isrf_small
    n = 4000
    eng = _engine(m)
    eng.set_schedule("warp")
    eng.enable_packet_log(n)
    eng.reset_tallies()
    eng.run(n, ipeel=ipeel)
    g = abi.packet_log_to_numpy(eng.packet_log(n))
    eng.close()
    _, lo = oracle_mod.run(abi.Bundle(m), n, ipeel=ipeel, nlog=n)
    o = abi.packet_log_to_numpy(lo)
    nodiff = (g["pad"] == 0) & (o["pad"] == 0)
    same, exact = _same_packets(g, o)
    ext = np.arange(1, n + 1) > n - int(round(0.3 * n))
    assert (o["i_orig"][ext] == 5).mean() > 0.3               # external packets ran
    assert exact[nodiff & ext].mean() >= 0.995 and exact[nodiff].mean() >= 0.995


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_isrf_wave_matches_warp_bitwise(isrf_small, precision):
    m = model.with_isrf(model.warm(model.small_2d()), 0.3)
    n = 3000
    logs = []
    for sched in ("warp", "wave"):
        eng = _engine(m, precision=precision)
        eng.set_schedule(sched)
        if sched == "wave":
            eng.set_wave_pool(512)
        eng.enable_packet_log(n)
        eng.reset_tallies()
        eng.run(n, ipeel=1)
        logs.append(abi.packet_log_to_numpy(eng.packet_log(n)))
        eng.close()
    for k in logs[0]:
        assert np.array_equal(logs[0][k], logs[1][k]), k

