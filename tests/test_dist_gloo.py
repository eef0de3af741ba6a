"""Multi-process packet sharding and the rank reduction, on CPU ranks (gloo).

Two processes each run the CPU oracle on their shard of one iteration and
sum their tallies with ``dist.allreduce_host_tallies`` -- the reference's
MPI_ALLREDUCE of newdisktherm_5_fuv.f90:520-604.  Since the shards are
contiguous ranges of one substream sequence, the sum must equal a single
run over the whole range: integer tallies exactly, FP64 sums up to summation
order, the REAL arrays to one rounding.
"""
import os
import socket
import tempfile

import numpy as np
import pytest

from src3_mpi_cfitsio_b200 import abi, dist, model

N_PACKETS = 1500


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _model():
    """The reduced 2-D model with every peel-off output on: image cubes,
    filter-band images and nested images."""
    return model.with_nested_images(model.with_filters(model.warm(model.small_2d())))


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as tdist
    from oracle import oracle
    tdist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        m = _model()
        lo, hi = dist.shard_range(N_PACKETS, rank, world)
        tal, _ = oracle.run(abi.Bundle(m), N_PACKETS, lo, hi, ipeel=1, threads=2)
        dist.allreduce_host_tallies(tal)
        if rank == 0:
            np.savez(os.path.join(out_dir, "reduced.npz"), **tal.arrays)
        tdist.barrier()
    finally:
        tdist.destroy_process_group()


@pytest.mark.parametrize("np_total,world", [(1, 1), (7, 2), (10, 3), (1000, 8), (2, 4), (123457, 5)])
def test_shard_range_partitions_the_packets(np_total, world):
    seen = []
    sizes = []
    for r in range(world):
        lo, hi = dist.shard_range(np_total, r, world)
        seen.extend(range(lo, hi + 1))
        sizes.append(hi - lo + 1)
    assert seen == list(range(1, np_total + 1))
    assert max(sizes) - min(sizes) <= 1


def test_two_gloo_ranks_reduce_to_the_single_run(oracle_mod):
    import torch.multiprocessing as mp
    world = 2
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_rank_main, args=(world, _free_port(), d), nprocs=world, join=True,
                           start_method="spawn")
        red = dict(np.load(os.path.join(d, "reduced.npz")))
    m = _model()
    one, _ = oracle_mod.run(abi.Bundle(m), N_PACKETS, ipeel=1, threads=2)
    ints = [k for k, a in one.arrays.items() if a.dtype in (np.int32, np.int64)]
    assert {"nabs", "dbig", "killed", "counters"} <= set(ints)
    for k in ints:
        assert np.array_equal(red[k], one[k]), k
    assert red["counters"][abi.COUNTERS.index("packets")] == N_PACKETS
    for k in ("dtauabs", "scalars"):
        assert np.allclose(red[k], one[k], rtol=1e-12, atol=0), k
    for k, a in one.arrays.items():
        if a.dtype == np.float32:
            assert np.allclose(red[k], a, rtol=2e-6, atol=1e-6 * max(1e-30, float(np.abs(a).max()))), k
    assert one["ti"].sum() > 0 and one["nums"].sum() > 0
    assert one["image_b_i"].sum() > 0 and one["image_ms_i"].sum() > 0


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shard_models_balances_whole_models(world):
    rng = np.random.default_rng(world)
    w = rng.uniform(1.0, 100.0, 64)
    parts = dist.shard_models(w, world)
    assert sorted(i for p in parts for i in p) == list(range(64))
    loads = [float(w[np.array(p, dtype=int)].sum()) for p in parts]
    assert max(loads) - min(loads) <= w.max() + 1e-9
    assert parts == dist.shard_models(w, world)          # deterministic


def _sweep_rank(rank, world, port, out_dir):
    import torch.distributed as tdist
    from oracle import oracle
    tdist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        models = _sweep_models()
        mine = dist.shard_models([m.ncells for m in models], world)[rank]
        for i in mine:
            tal, _ = oracle.run(abi.Bundle(models[i]), 300, ipeel=0, threads=1)
            np.savez(os.path.join(out_dir, f"model{i}.npz"), nabs=tal["nabs"], counters=tal["counters"],
                     dtauabs=tal["dtauabs"])
        tdist.barrier()
    finally:
        tdist.destroy_process_group()


def _sweep_models():
    return [model.warm(model.small_2d(nrg=n, ntg=t, npg=p, massd=md))
            for n, t, p, md in ((21, 15, 2, 1e-3), (27, 17, 4, 3e-3), (31, 21, 2, 1e-2), (25, 13, 3, 5e-4))]


def test_two_gloo_ranks_run_a_sharded_sweep(oracle_mod):
    """A sweep sharded by whole models over two ranks gives every model the
    result of its own single-process run (no exchange between ranks)."""
    import torch.multiprocessing as mp
    world = 2
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_sweep_rank, args=(world, _free_port(), d), nprocs=world, join=True,
                           start_method="spawn")
        got = [dict(np.load(os.path.join(d, f"model{i}.npz"))) for i in range(4)]
    for i, m in enumerate(_sweep_models()):
        one, _ = oracle_mod.run(abi.Bundle(m), 300, ipeel=0, threads=1)
        assert np.array_equal(got[i]["nabs"], one["nabs"]) and np.array_equal(got[i]["counters"], one["counters"])
        assert np.allclose(got[i]["dtauabs"], one["dtauabs"], rtol=1e-12, atol=0)
