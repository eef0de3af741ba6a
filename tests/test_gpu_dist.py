"""Rank reduction of the tallies on the GPU (newdisktherm_5_fuv.f90:520-604).

* ``mcrt_accumulate_tallies`` adds downloaded tallies back into the device;
* ``mcrt_device_tallies_view`` exposes the device tally buffer for an
  in-place NCCL all-reduce (a one-rank NCCL group here: one GPU per test);
* two contexts that run the two shards of one iteration, reduced and
  refreshed, give the temperature of one context that ran the whole range.
"""
import os
import tempfile

import numpy as np
import pytest

from src3_mpi_cfitsio_b200 import dist, model

pytestmark = pytest.mark.gpu


def _engine(m, precision="fp64"):
    from src3_mpi_cfitsio_b200.engine import Engine
    return Engine(m, precision=precision)


@pytest.fixture(scope="module")
def warm_small():
    return model.warm(model.small_2d())


def _close(a, b, k):
    x, y = a[k].astype(np.float64), b[k].astype(np.float64)
    assert np.allclose(x, y, rtol=1e-6, atol=1e-6 * max(1e-30, float(np.abs(y).max()))), k


def test_accumulate_adds_host_tallies(warm_small):
    eng = _engine(warm_small)
    eng.reset_tallies()
    eng.run(2000, ipeel=1)
    a = eng.download()
    eng.reset_tallies()
    eng.accumulate(a)
    eng.accumulate(a)
    b = eng.download()
    for k, x in a.arrays.items():
        if x.dtype in (np.int32, np.int64):
            assert np.array_equal(b[k], 2 * x), k
        else:
            assert np.allclose(b[k], 2 * x.astype(np.float64), rtol=1e-6, atol=0), k
    eng.close()


def test_device_view_aliases_the_tallies_and_reduces_with_nccl(warm_small):
    import torch
    import torch.distributed as tdist
    eng = _engine(warm_small)
    eng.reset_tallies()
    eng.run(2000, ipeel=1)
    a = eng.download()
    f64, u64, i32 = dist.device_tally_tensors(eng)
    nc = eng.cfg.nrg * eng.cfg.ntg * eng.cfg.npg
    assert np.array_equal(f64[:nc].cpu().numpy(), a["dtauabs"])
    assert np.array_equal(i32[:nc].cpu().numpy(), a["nabs"])
    assert np.array_equal(u64.cpu().numpy(), a["counters"])
    with tempfile.TemporaryDirectory() as d:
        store = tdist.FileStore(os.path.join(d, "store"), 1)
        tdist.init_process_group("nccl", store=store, rank=0, world_size=1)
        try:
            dist.allreduce_device_tallies(eng)          # one rank: the sum is the identity
            b = eng.download()
            for k in ("dtauabs", "nabs", "counters", "si", "ti", "image_m_i"):
                assert np.array_equal(b[k], a[k]), k
            for t in (f64, u64, i32):                    # the views are the engine's buffer
                t.mul_(3)
            torch.cuda.synchronize()
            c = eng.download()
            assert np.array_equal(c["nabs"], 3 * a["nabs"])
            assert np.array_equal(c["counters"], 3 * a["counters"])
            assert np.allclose(c["dtauabs"], 3 * a["dtauabs"], rtol=1e-15, atol=0)
        finally:
            tdist.destroy_process_group()
    eng.close()


@pytest.mark.parametrize("path,diffusion", [("host", False), ("device", False), ("device", True)])
def test_two_shards_reduce_to_the_single_run(warm_small, path, diffusion):
    """Two contexts run the two shards of one iteration; their tallies are
    summed either on the host (download, sum, reset, accumulate) or on the
    device (the tally views summed into both buffers, which is what an NCCL
    all-reduce over two GPUs leaves in each); then the diffusion refresh and
    tfinal.  Without diffusion the result equals one context over the whole
    range up to summation order.  With diffusion, each shard emitted from
    diffusion surfaces with its own absorption count (as each MPI rank heats
    a private copy in the reference), so the temperatures agree within the
    Monte Carlo noise."""
    import torch
    m = model.with_diffusion(warm_small) if diffusion else warm_small
    n = 6000
    one = _engine(m)
    one.reset_tallies()
    one.run(n, ipeel=0)
    t_one = one.download(images=False)
    one.refresh_diffusion()
    td_one, _, _ = one.update_temperature(n, 1)
    shards = []
    for r in range(2):
        e = _engine(m)
        lo, hi = dist.shard_range(n, r, 2)
        e.reset_tallies()
        e.run(n, lo, hi, ipeel=0)
        shards.append(e)
    if path == "host":
        total = shards[0].download(images=False).add_(shards[1].download(images=False))
        for e in shards:
            e.reset_tallies()
            e.accumulate(total)
    else:
        views = [dist.device_tally_tensors(e) for e in shards]
        for e in shards:
            e.synchronize()
        for seg in range(3):
            s = views[0][seg] + views[1][seg]
            for v in views:
                v[seg].copy_(s)
        torch.cuda.synchronize()
    temps = []
    for e in shards:
        e.refresh_diffusion()
        td, _, _ = e.update_temperature(n, 1)
        temps.append(td)
        red = e.download(images=False)
        if not diffusion:
            for k in ("nabs", "dbig", "killed"):
                assert np.array_equal(red[k], t_one[k]), k
            assert np.allclose(red["dtauabs"], t_one["dtauabs"], rtol=1e-12, atol=1e-300)
            _close(red, t_one, "si")
            assert red.counters()["packets"] == n
    assert np.array_equal(temps[0], temps[1])            # every rank ends with the same temperature
    if not diffusion:
        assert np.allclose(temps[0], td_one, rtol=1e-9, atol=0)
    else:
        rel = np.abs(temps[0] / td_one - 1.0)
        assert np.median(rel) < 1e-2 and np.quantile(rel, 0.9) < 0.1
    for e in shards + [one]:
        e.close()
