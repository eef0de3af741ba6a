// mcrt_mixed.cu -- mixed-precision transport build.
//
// The transport and peel-off kernels of mcrt_sched.cuh / mcrt_peel.cuh
// compiled with MCRT_MIXED:
//  * the packet walk and the peel-off walk run in FP32 in the
//    closest-approach form (QRay, mcrt_transport.cuh): cone and plane roots,
//    cell opacities and the walk state in FP32; sphere roots in FP64 where
//    a wall borders a cell thinner than 1 % of its radius (the disk rim);
//    the along-ray coordinate, the cumulative optical depth, its comparison
//    with the sampled tau, and every tally in FP64;
//  * scattering (rejection sampling, frame rotations, the peel-off phase
//    matrix) in FP32.
// Packet positions between walks, directions, frequencies and the event
// code stay FP64.  The device code is compiled into its own namespace so
// that it can coexist with the FP64 build's kernels; the launch parameters
// have the same layout.
#include <cuda_runtime.h>

#define MCRT_MIXED 1
// The FP32 walk kernel runs 8 blocks (32 warps) per SM at <= 64 registers:
// 1.33x the walk rate of 4 blocks on the 1e8-packet 2-D iteration.
#ifndef MCRT_WALK_MIN_BLOCKS
#define MCRT_WALK_MIN_BLOCKS 8
#endif
// The peel-off kernel at 4 blocks (16 warps) per SM, <= 128 registers: the
// phase-matrix and binning code spills about 200 B to local memory, but the
// FP32 walk it shares the kernel with runs a third more warps.  B200, mixed,
// peeled iterations: 2-D 1e7 packets 1141 -> 824 ms, 3-D clumpy 2e6 packets
// 1118 -> 950 ms (interleaved on one box); 5 blocks (<= 102 registers,
// ~600 B spilled) was slower than 3.
#ifndef MCRT_PEEL_MIN_BLOCKS
#define MCRT_PEEL_MIN_BLOCKS 4
#endif
#define mcrt mcrt_mixed
#include "mcrt_sched.cuh"
#include "mcrt_peel.cuh"
#include "mcrt_wave.cuh"
#include "mcrt_batch.cuh"
#undef mcrt

namespace mcrt {
struct LaunchParams;
struct WaveArgs;
struct BatchItem;

cudaError_t launch_batch_mixed(const LaunchParams* params, const BatchItem* items, int64_t nitems,
                               unsigned long long* item_next, unsigned long long* chunk_next, int32_t event_batch,
                               int grid, cudaStream_t s) {
  mcrt_mixed::transport_batch<<<grid, mcrt_mixed::kBlock, 0, s>>>(
      reinterpret_cast<const mcrt_mixed::LaunchParams*>(params), reinterpret_cast<const mcrt_mixed::BatchItem*>(items),
      nitems, item_next, chunk_next, event_batch);
  return cudaGetLastError();
}

int batch_mixed_blocks_per_sm() {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, mcrt_mixed::transport_batch, mcrt_mixed::kBlock, 0) != cudaSuccess) return 1;
  return n > 0 ? n : 1;
}

cudaError_t launch_wave_event_mixed(const LaunchParams& p, const WaveArgs& w, int grid, cudaStream_t s) {
  const auto& q = reinterpret_cast<const mcrt_mixed::LaunchParams&>(p);
  const auto& v = reinterpret_cast<const mcrt_mixed::WaveArgs&>(w);
  mcrt_mixed::wave_event<<<grid, mcrt_mixed::kBlock, 0, s>>>(q, v);
  return cudaGetLastError();
}

cudaError_t launch_wave_walk_mixed(const LaunchParams& p, const WaveArgs& w, int grid, cudaStream_t s) {
  const auto& q = reinterpret_cast<const mcrt_mixed::LaunchParams&>(p);
  const auto& v = reinterpret_cast<const mcrt_mixed::WaveArgs&>(w);
  mcrt_mixed::wave_walk<<<grid, mcrt_mixed::kBlock, 0, s>>>(q, v);
  return cudaGetLastError();
}

cudaError_t launch_wave_tail_mixed(const LaunchParams& p, const WaveArgs& w, int grid, cudaStream_t s) {
  const auto& q = reinterpret_cast<const mcrt_mixed::LaunchParams&>(p);
  const auto& v = reinterpret_cast<const mcrt_mixed::WaveArgs&>(w);
  mcrt_mixed::wave_tail<<<grid, mcrt_mixed::kBlock, 0, s>>>(q, v);
  return cudaGetLastError();
}

int wave_tail_mixed_blocks_per_sm() {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, mcrt_mixed::wave_tail, mcrt_mixed::kBlock, 0) != cudaSuccess) return 1;
  return n > 0 ? n : 1;
}

int wave_event_mixed_blocks_per_sm() {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, mcrt_mixed::wave_event, mcrt_mixed::kBlock, 0) != cudaSuccess) return 1;
  return n > 0 ? n : 1;
}

int wave_walk_mixed_blocks_per_sm() {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, mcrt_mixed::wave_walk, mcrt_mixed::kBlock, 0) != cudaSuccess) return 1;
  return n > 0 ? n : 1;
}

cudaError_t launch_transport_mixed(const LaunchParams& p, int grid, cudaStream_t s) {
  const auto& q = reinterpret_cast<const mcrt_mixed::LaunchParams&>(p);
  mcrt_mixed::transport_sched<<<grid, mcrt_mixed::kBlock, 0, s>>>(q);
  return cudaGetLastError();
}

int transport_mixed_blocks_per_sm() {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, mcrt_mixed::transport_sched, mcrt_mixed::kBlock, 0) != cudaSuccess) return 1;
  return n > 0 ? n : 1;
}

cudaError_t launch_peel_mixed(const LaunchParams& p, unsigned long long* next_item, int grid, cudaStream_t s) {
  const auto& q = reinterpret_cast<const mcrt_mixed::LaunchParams&>(p);
  mcrt_mixed::peel_sched<<<grid, mcrt_mixed::kBlock, 0, s>>>(q, next_item);
  return cudaGetLastError();
}

int peel_mixed_blocks_per_sm() {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, mcrt_mixed::peel_sched, mcrt_mixed::kBlock, 0) != cudaSuccess) return 1;
  return n > 0 ? n : 1;
}

}  // namespace mcrt
