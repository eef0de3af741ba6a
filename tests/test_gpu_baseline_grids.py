"""Parity on the benchmark's own grids (not the reduced test grids).

* FP64 engine vs the CPU oracle, packet for packet, on the 2-D benchmark
  model at its converged Lucy temperature (rim-refined walls, the disk
  interior under the diffusion treatment), with and without peel-offs, and
  on the full 3-D clumpy grid (200 x 199 x 64 cells) with tabulated Mueller
  matrices.  Packets that reach a diffusion cell depend on the order of the
  surface heating (the reference's result depends on its rank count for the
  same reason) and are compared as an ensemble.
* Mixed build vs FP64 build with independent random streams at equal packet
  counts: chi^2 per SED and peeled-SED bin from the tallies' own variance
  arrays (si2, ti2), image differences against the FP64-vs-FP64 noise floor,
  and cell temperatures within 0.5 % where the Monte Carlo error allows it.
"""
import copy

import numpy as np
import pytest

from src3_mpi_cfitsio_b200 import abi, model

pytestmark = pytest.mark.gpu

SEEDS = [(12345678, 87654321), (23456789, 98765432), (34567891, 19876543)]


def _engine(m, precision="fp64"):
    from src3_mpi_cfitsio_b200.engine import Engine
    return Engine(m, precision=precision)


def _same_packets(g, o):
    same = ((g["ndraws"] == o["ndraws"]) & (g["nscat"] == o["nscat"]) & (g["nabs"] == o["nabs"]) &
            (g["status"] == o["status"]) & (g["ncross"] == o["ncross"]) & (g["nstar"] == o["nstar"]))
    close = np.isclose(g["nub"], o["nub"], rtol=1e-9, atol=0) & np.isclose(g["sip"], o["sip"], rtol=1e-9, atol=1e-12)
    return same & close


@pytest.fixture(scope="module")
def bench2d():
    return model.reference_2d_converged()


@pytest.mark.parametrize("ipeel,n", [(0, 20000), (1, 3000)])
def test_fp64_event_for_event_on_the_benchmark_grid(bench2d, oracle_mod, ipeel, n):
    m = bench2d
    assert (m.grid["diffus"] > 0).any()
    eng = _engine(m)
    eng.enable_packet_log(n)
    eng.reset_tallies()
    eng.run(n, ipeel=ipeel)
    g = abi.packet_log_to_numpy(eng.packet_log(n))
    tg = eng.download(images=False)
    eng.close()
    to, lo = oracle_mod.run(abi.Bundle(m), n, ipeel=ipeel, nlog=n, images=False)
    o = abi.packet_log_to_numpy(lo)
    nodiff = (g["pad"] == 0) & (o["pad"] == 0)
    assert nodiff.mean() > 0.5
    exact = _same_packets(g, o)
    assert exact[nodiff].mean() >= 0.995, exact[nodiff].mean()
    assert (g["status"] == 3).sum() == 0
    cg, co = tg.counters(), to.counters()
    assert cg["packets"] == co["packets"] == n
    assert abs(cg["crossings"] - co["crossings"]) <= 0.02 * co["crossings"]
    a = tg.shaped("nums")[..., 0].sum(axis=(1, 2, 3))
    b = to.shaped("nums")[..., 0].sum(axis=(1, 2, 3))
    assert np.all(np.abs(a - b) <= 5 * np.sqrt(np.maximum(b, 1)) + 5)
    if ipeel:
        # every event adds 10 inclinations x 3 components to numt, so its
        # Monte Carlo spread (from the diffusion packets) is far above Poisson
        x, y = tg["numt"].astype(np.float64), to["numt"].astype(np.float64)
        assert abs(x.sum() - y.sum()) <= 0.05 * y.sum()


def test_fp64_event_for_event_on_the_clumpy_grid(oracle_mod):
    """The full 3-D clumpy grid (201 x 199 x 65 walls, fractal clumps, phi
    planes) with tabulated S11-S44 scattering, peel-offs to 20 inclinations
    (peeled SED; the image cubes are left out to keep the oracle's host
    memory small)."""
    m = model.with_diffusion(model.warm(model.with_mueller(model.clumpy_3d())))
    m.config["output_imcube"] = 0
    n = 2000
    eng = _engine(m)
    eng.enable_packet_log(n)
    eng.reset_tallies()
    eng.run(n, ipeel=1)
    g = abi.packet_log_to_numpy(eng.packet_log(n))
    tg = eng.download(images=False)
    eng.close()
    to, lo = oracle_mod.run(abi.Bundle(m), n, ipeel=1, nlog=n, images=False)
    o = abi.packet_log_to_numpy(lo)
    nodiff = (g["pad"] == 0) & (o["pad"] == 0)
    exact = _same_packets(g, o)
    assert exact[nodiff].mean() >= 0.995, exact[nodiff].mean()
    assert (g["status"] == 3).sum() == 0
    cg, co = tg.counters(), to.counters()
    assert cg["peel_cross"] > 1000 * n
    # the diffusion packets (a few, with many events each) differ only
    # statistically, so the aggregates carry their Monte Carlo noise
    assert abs(cg["peel_cross"] - co["peel_cross"]) <= 0.1 * co["peel_cross"]
    x, y = tg["ti"].astype(np.float64), to["ti"].astype(np.float64)
    assert abs(x.sum() - y.sum()) <= 0.05 * abs(y.sum())


def _run(m, prec, n, seeds, ipeel, images=False):
    eng = _engine(m, prec)
    eng.reset_tallies()
    eng.run(n, iteration=2, ipeel=ipeel, seeds=seeds)
    tal = eng.download(images=images)
    td, _, _ = eng.update_temperature(n, 2) if not ipeel else (None, None, None)
    c = tal.counters()
    eng.close()
    return tal, td, c


def _chi2(a, b, k, k2, minn):
    """chi^2 per degree of freedom of two independent tallies of sums k with
    per-bin sums of squares k2, over bins where both have >= minn packets."""
    cnt = "nums" if k.startswith("s") else "numt"
    n1, n2 = a[cnt].astype(np.float64), b[cnt].astype(np.float64)
    x, y = a[k].astype(np.float64), b[k].astype(np.float64)
    v = a[k2].astype(np.float64) + b[k2].astype(np.float64)
    use = (n1 >= minn) & (n2 >= minn) & (v > 0)
    return float(((x - y)[use] ** 2 / v[use]).sum() / max(use.sum(), 1)), int(use.sum())


def test_mixed_vs_fp64_chi2_with_independent_seeds(bench2d):
    """SED and peeled SED, 4e6 / 2e6 packets per run: mixed (seed set C)
    against FP64 (seed set A) has chi^2 per bin ~ 1, like FP64 (B) against
    FP64 (A); the images' L1 distance stays at the FP64-vs-FP64 noise floor."""
    m = bench2d
    a, _, ca = _run(m, "fp64", 4_000_000, SEEDS[0], 0)
    b, _, _ = _run(m, "fp64", 4_000_000, SEEDS[1], 0)
    c, _, cc = _run(m, "mixed", 4_000_000, SEEDS[2], 0)
    assert cc["geom_fail"] == 0 and cc["packets"] == 4_000_000
    assert abs(cc["crossings"] - ca["crossings"]) <= 0.002 * ca["crossings"]
    # The FP64-vs-FP64 chi^2 calibrates the test: within an iteration the
    # diffusion surfaces heat with every absorption, which couples packets
    # and spreads the SED beyond independent sampling (the reference has the
    # same coupling); mixed-vs-FP64 must show no excess beyond that.
    ctrl, dof = _chi2(a, b, "si", "si2", 30)
    mix, dof2 = _chi2(a, c, "si", "si2", 30)
    assert dof > 200 and dof2 > 200
    assert mix <= ctrl * (1.0 + 4.0 * np.sqrt(2.0 / dof2)) + 0.05, (mix, ctrl, dof2)
    pa, _, _ = _run(m, "fp64", 2_000_000, SEEDS[0], 1, images=True)
    pb, _, _ = _run(m, "fp64", 2_000_000, SEEDS[1], 1, images=True)
    pc, _, _ = _run(m, "mixed", 2_000_000, SEEDS[2], 1, images=True)
    ctrl, dof = _chi2(pa, pb, "ti", "ti2", 30)
    mix, dof2 = _chi2(pa, pc, "ti", "ti2", 30)
    assert dof2 > 100
    assert mix <= max(ctrl, 1.0) * (1.0 + 4.0 * np.sqrt(2.0 / dof2)) + 0.05, (mix, ctrl, dof2)
    for k in ("image_m_i", "image_m_q"):
        x, y, z = (t[k].astype(np.float64) for t in (pa, pb, pc))
        floor = np.abs(x - y).sum()
        assert np.abs(x - z).sum() <= 1.15 * floor, (k, np.abs(x - z).sum() / floor)


def test_mixed_vs_fp64_temperatures_within_half_a_percent(bench2d):
    """Cell temperatures after tfinal from 1e8-packet iterations with
    independent streams: in cells with >= 5e4 absorptions (Monte Carlo
    error of T ~0.1 % per run) the mixed build's temperatures are within
    0.5 % of the FP64 build's in 95 % of the cells, unbiased to 0.05 %, and
    spread no wider than FP64 against itself."""
    m = bench2d
    a, ta, _ = _run(m, "fp64", 100_000_000, SEEDS[0], 0)
    b, tb, _ = _run(m, "fp64", 100_000_000, SEEDS[1], 0)
    c, tc, _ = _run(m, "mixed", 100_000_000, SEEDS[2], 0)
    good = (a["nabs"] >= 50000) & (c["nabs"] >= 50000) & (ta > 2.0 / 11605.0)
    assert good.sum() > 500, good.sum()
    rel_mix = np.abs(tc[good] / ta[good] - 1.0)
    rel_ctl = np.abs(tb[good] / ta[good] - 1.0)
    q95m, q95c = np.quantile(rel_mix, 0.95), np.quantile(rel_ctl, 0.95)
    assert q95m <= 0.005, (q95m, q95c, good.sum())
    assert abs(np.median(tc[good] / ta[good] - 1.0)) <= 5e-4
    assert q95m <= 1.3 * q95c + 2e-4, (q95m, q95c)
