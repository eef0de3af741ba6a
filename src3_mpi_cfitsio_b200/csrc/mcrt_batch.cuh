// mcrt_batch.cuh -- many models in one persistent launch.
//
// A batch of models (contexts of uneven grids, tables and packet counts)
// runs one Lucy iteration's packet loop (the reference's `disk` loop,
// newdisktherm_5_fuv.f90:220-491, without peel-offs) in a single launch.
// The work is a list of (model, packet chunk) items taken from a global
// counter by whole warps.  A warp copies the item's model parameters
// (LaunchParams: the model view, its tallies, the packet split and streams)
// into its own shared-memory slot and runs the warp-scheduled loop of
// mcrt_sched.cuh over the chunk, then takes the next item.  Warps never wait
// for one another (no block barrier), so a warp held by a long history in an
// optically thick model does not stall the rest of its block, and small and
// large models share the GPU.
// Every packet keeps its own substream (block (iter-1)*np + iphot-1 of its
// model), so each model's histories are the same as in a run of its own.
#pragma once
#include "mcrt_sched.cuh"

namespace mcrt {

__global__ void __launch_bounds__(kBlock, MCRT_SCHED_MIN_BLOCKS)
transport_batch(const LaunchParams* __restrict__ params, const BatchItem* __restrict__ items, int64_t nitems,
                unsigned long long* item_next, unsigned long long* chunk_next, int32_t event_batch) {
  constexpr unsigned FULL = 0xffffffffu;
  __shared__ double spec[5 * kMaxSlot * kBlock];
  __shared__ LaunchParams Ps[kBlock / 32];
  const int lane = threadIdx.x & 31;
  LaunchParams& P = Ps[threadIdx.x >> 5];
  for (;;) {
    unsigned long long k = 0;
    if (lane == 0) k = atomicAdd(item_next, 1ull);
    const int64_t it = (int64_t)__shfl_sync(FULL, k, 0);
    if (it >= nitems) break;                   // uniform over the warp
    const BatchItem B = items[it];
    {   // the item's model parameters into this warp's shared slot
      const uint32_t* src = reinterpret_cast<const uint32_t*>(params + B.model);
      uint32_t* dst = reinterpret_cast<uint32_t*>(&P);
      for (int w = lane; w < (int)(sizeof(LaunchParams) / 4); w += 32) dst[w] = src[w];
    }
    __syncwarp();
    if (lane == 0) {
      P.lo = B.lo;
      P.hi = B.hi;
      P.next = chunk_next + it;                // this chunk's packet counter
      P.log_off = B.lo - 1;                    // log entries by packet number
      P.event_batch = event_batch;
    }
    __syncwarp();
    {
      Lane L(P.m, P.t, spec);
      warp_loop(L, P);
    }
    __syncwarp();                              // P is rewritten by the next item
  }
}

}  // namespace mcrt
