"""Batched models (mcrt_batch_*): one launch per iteration over many uneven
models gives each model the results of its own run.

Every packet of model i draws block (iter-1)*np[i] + iphot-1 of the stream,
as in a run of model i alone, and the batch kernel steps it through the same
warp-scheduled loop: packet logs agree bit for bit with the warp schedule's,
counters exactly, FP64 tallies up to summation order.
"""
import numpy as np
import pytest

from src3_mpi_cfitsio_b200 import abi, model

pytestmark = pytest.mark.gpu


def _uneven():
    """Three small models of different grids, wavelength sets and densities
    (one 3-D)."""
    a = model.warm(model.small_2d())
    b = model.warm(model.small_2d(nrg=41, ntg=25, npg=2, nlambda=70, massd=0.002, thet1_deg=30.0))
    c = model.warm(model.small_2d(nrg=27, ntg=17, npg=7, nlambda=55, rate=3e-6))
    return [a, b, c]


@pytest.fixture(scope="module")
def uneven():
    return _uneven()


def _engine(m, precision):
    from src3_mpi_cfitsio_b200.engine import Engine
    e = Engine(m, precision=precision)
    e.set_schedule("warp", 16)
    return e


def _single(models, nps, precision, iteration, nlog):
    out = []
    for m, n in zip(models, nps):
        e = _engine(m, precision)
        e.enable_packet_log(nlog)
        e.reset_tallies()
        e.run(n, ipeel=0, iteration=iteration)
        tal = e.download(images=False)
        log = abi.packet_log_to_numpy(e.packet_log(nlog))
        td, _, _ = e.update_temperature(n, iteration)
        out.append((log, tal, td))
        e.close()
    return out


def _compare(ref, got):
    for (la, ta, tda), (lb, tb, tdb) in zip(ref, got):
        for k in la:
            assert np.array_equal(la[k], lb[k]), k
        ca, cb = ta.counters(), tb.counters()
        for k in ("packets", "crossings", "interactions", "scatters", "geom_fail", "resets", "killed", "exited",
                  "starhits"):
            assert ca[k] == cb[k], k
        for k in ("nabs", "dbig", "dsg", "killed"):
            assert np.array_equal(ta[k], tb[k]), k
        for k in ("si", "nums", "dtauabs"):
            x, y = ta[k], tb[k]
            assert np.allclose(x, y, rtol=1e-9, atol=1e-12 * max(1e-30, float(np.abs(x).max()))), k
        assert np.allclose(tda, tdb, rtol=1e-9, atol=0)


@pytest.mark.parametrize("schedule,precision", [("persistent", "fp64"), ("persistent", "mixed"), ("wave", "fp64"),
                                                ("wave", "mixed")])
def test_batch_matches_single_runs(uneven, schedule, precision):
    from src3_mpi_cfitsio_b200.batch import Batch
    nps = [3000, 1700, 2200]
    nlog = 1700
    ref = _single(uneven, nps, precision, 2, nlog)
    engines = [_engine(m, precision) for m in uneven]
    for e in engines:
        e.enable_packet_log(nlog)
    b = Batch(engines)
    b.set_tuning(0, 16, 3)                   # several chunks per model
    b.set_schedule(schedule, 512)            # several waves per model
    b.run_iteration(nps, iteration=2)
    assert b.kernel_ms() > 0
    got = []
    for e, n in zip(engines, nps):
        tal = e.download(images=False)
        log = abi.packet_log_to_numpy(e.packet_log(nlog))
        td, _, _ = e.update_temperature(n, 2)
        got.append((log, tal, td))
    _compare(ref, got)
    b.close()
    for e in engines:
        e.close()


@pytest.mark.parametrize("schedule", ["persistent", "wave"])
def test_batch_with_diffusion_cells(uneven, schedule):
    """A model with diffusion cells in the batch: packets that never reach a
    diffusion cell stay bit-equal to its own run, the diffusion count agrees
    within Monte Carlo error (the surface cells heat in arrival order), and
    the other model of the batch is untouched by it."""
    from src3_mpi_cfitsio_b200.batch import Batch
    models = [model.with_diffusion(model.warm(model.small_2d())), uneven[1]]
    nps = [20000, 3000]
    nlog = 3000
    ref = _single(models, nps, "fp64", 2, 20000)
    engines = [_engine(m, "fp64") for m in models]
    engines[0].enable_packet_log(20000)
    engines[1].enable_packet_log(nlog)
    b = Batch(engines)
    b.set_tuning(0, 16, 2)
    b.set_schedule(schedule, 4096)
    b.run_iteration(nps, iteration=2)
    got = []
    for e, n, nl in zip(engines, nps, (20000, nlog)):
        tal = e.download(images=False)
        log = abi.packet_log_to_numpy(e.packet_log(nl))
        td, _, _ = e.update_temperature(n, 2)
        got.append((log, tal, td))
    g, o = got[0][0], ref[0][0]
    nodiff = (g["pad"] == 0) & (o["pad"] == 0)
    assert o["pad"].sum() > 20
    for k in ("ndraws", "nscat", "nabs", "status", "ncross"):
        assert (g[k] == o[k])[nodiff].mean() >= 0.995, k
    dg, do = g["pad"].sum(), o["pad"].sum()
    assert abs(dg - do) <= 5 * np.sqrt(do) + 5
    _compare([(_head(ref[1][0], nlog), ref[1][1], ref[1][2])], [got[1]])
    b.close()
    for e in engines:
        e.close()


def _head(log, n):
    return {k: v[:n] for k, v in log.items()}


@pytest.mark.parametrize("schedule", ["persistent", "wave"])
def test_batch_graph_replay_and_recapture(uneven, schedule):
    """The same packet counts replay the captured graph (tallies are reset
    inside it, the iteration's random blocks are read from device memory);
    new counts re-capture it."""
    from src3_mpi_cfitsio_b200.batch import Batch
    engines = [_engine(m, "mixed") for m in uneven]
    b = Batch(engines)
    b.set_schedule(schedule, 1000)
    res = []
    runs = (([2000, 1000, 1500], 1), ([2000, 1000, 1500], 1), ([900, 2100, 1200], 1), ([2000, 1000, 1500], 2))
    for nps, it in runs:
        b.run_iteration(nps, iteration=it)
        res.append([e.download(images=False) for e in engines])
    for k in ("nabs", "dbig"):
        for i in range(3):
            assert np.array_equal(res[0][i][k], res[1][i][k]), k
    for i, n in enumerate([900, 2100, 1200]):
        assert res[2][i].counters()["packets"] == n
    # the replayed graph at iteration 2 = a single run at iteration 2
    ref = _single(uneven[1:2], [1000], "mixed", 2, 1)
    assert np.array_equal(res[3][1]["nabs"], ref[0][1]["nabs"])
    assert not np.array_equal(res[3][1]["nabs"], res[0][1]["nabs"])
    b.close()
    for e in engines:
        e.close()


def test_batch_tuner_choice(uneven):
    from src3_mpi_cfitsio_b200.batch import Batch
    engines = [_engine(m, "mixed") for m in uneven]
    b = Batch(engines)
    t = b.tune(600)
    assert t["schedule"] in ("persistent", "wave")
    assert t["blocks_per_sm"] >= 1 and 1 <= t["event_batch"] <= 32 and t["items_per_warp"] >= 1
    assert t["wave_slots"] >= 64
    b.run_iteration([700, 800, 900])
    for e, n in zip(engines, (700, 800, 900)):
        assert e.download(images=False).counters()["packets"] == n
    b.close()
    for e in engines:
        e.close()


def test_batch_rejects_mixed_precisions(uneven):
    from src3_mpi_cfitsio_b200.batch import Batch
    from src3_mpi_cfitsio_b200.engine import MCRTError
    e1 = _engine(uneven[1], "fp64")
    e2 = _engine(uneven[2], "mixed")
    with pytest.raises(MCRTError):
        Batch([e1, e2])
    e1.close()
    e2.close()
