"""Multi-process runs: packet shards and the rank reduction of the tallies.

The reference runs one MPI rank per core, each with its own random generator
and np/numprocs packets, and sums every tally over the ranks with
MPI_ALLREDUCE (newtts.f90:104-105, 139; newdisktherm_5_fuv.f90:520-604).
Here the ranks are GPUs (one process each, torch.distributed) and split ONE
iteration's packet range into contiguous shards of the same substream
sequence, so the summed tallies equal a one-GPU run of the whole range
whatever the number of ranks.

A batched sweep (``batch.Batch``) shards whole models instead
(``shard_models``): its models are independent, so no tally crosses ranks.

Two reductions:

* ``allreduce_device_tallies`` sums the device tally buffer in place over
  the process group (NCCL on GPUs; no host round trip);
* ``allreduce_host_tallies`` sums downloaded host arrays (any backend, gloo
  on CPU); ``Engine.accumulate`` puts the sum back on the device.

After either, ``Engine.refresh_diffusion`` recomputes the diffusion cells'
temperature from the summed absorption counts and ``Engine.update_temperature``
runs ``tfinal`` on the summed ``dtauabs``.
"""
from __future__ import annotations

import numpy as np


def shard_range(np_total: int, rank: int, world: int) -> tuple[int, int]:
    """1-based inclusive packet range of `rank`: contiguous, disjoint, covering
    1..np_total, sizes differing by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    base, extra = divmod(int(np_total), world)
    lo = rank * base + min(rank, extra) + 1
    hi = lo + base - 1 + (1 if rank < extra else 0)
    return lo, hi


def shard_models(weights, world: int) -> list:
    """Models of a batched sweep per rank (no exchange between ranks: every
    model is whole on one GPU).  Greedy longest-first assignment by `weights`
    (e.g. packets x cells per model) to the least-loaded rank, ties to the
    lower rank: deterministic, and the heaviest rank carries at most the
    lightest one's load plus one model.  Returns one ascending index list
    per rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    w = [float(x) for x in weights]
    order = sorted(range(len(w)), key=lambda i: (-w[i], i))
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += w[i]
    return [sorted(x) for x in out]


class _DeviceArray:
    """A device buffer described by __cuda_array_interface__ (for torch.as_tensor)."""

    def __init__(self, ptr: int, n: int, typestr: str, device: int):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}
        self.device = device


def device_tally_tensors(engine, device: int = 0):
    """torch views (no copy) of the engine's device tally segments."""
    import torch
    v = engine.device_tallies()
    dev = torch.device("cuda", device)
    out = []
    for ptr, n, ts in ((v.f64, v.n_f64, "<f8"), (v.u64, v.n_u64, "<i8"), (v.i32, v.n_i32, "<i4")):
        out.append(torch.as_tensor(_DeviceArray(ptr, n, ts, device), device=dev))
    return out


def allreduce_device_tallies(engine, group=None, device: int = 0):
    """Sum the device tallies of every rank in place (the MPI_ALLREDUCE block)."""
    import torch
    import torch.distributed as dist
    engine.synchronize()                 # the engine's stream has finished writing the tallies
    for t in device_tally_tensors(engine, device):
        if t.numel():
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    torch.cuda.synchronize(device)       # the sums are complete before the engine's stream reads them


def allreduce_host_tallies(tal, group=None):
    """Sum downloaded tallies (abi.TallyArrays) over the ranks, in place.

    Integer and FP64 arrays are summed exactly in their own type; the REAL
    (FP32) SED/image arrays are summed in FP64 and rounded once."""
    import torch
    import torch.distributed as dist
    for name, a in tal.arrays.items():
        if a.dtype == np.float32:
            t = torch.from_numpy(a.astype(np.float64))
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
            a[:] = t.numpy().astype(np.float32)
        else:
            t = torch.from_numpy(a)
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)


def run_sharded_iteration(engine, np_total: int, iteration: int, *, ipeel: int = 0, group=None,
                          device: int = 0, rank: int | None = None, world: int | None = None):
    """One Lucy iteration over all ranks: this rank's packet shard, device
    all-reduce of the tallies, diffusion refresh.  Returns (lo, hi)."""
    import torch.distributed as dist
    rank = dist.get_rank(group) if rank is None else rank
    world = dist.get_world_size(group) if world is None else world
    lo, hi = shard_range(np_total, rank, world)
    engine.reset_tallies()
    if hi >= lo:
        engine.run(np_total, lo, hi, iteration=iteration, ipeel=ipeel)
    allreduce_device_tallies(engine, group, device)
    if hi >= lo:                         # a rank with an empty shard (np_total < world) keeps its temperature
        engine.refresh_diffusion()
    return lo, hi
