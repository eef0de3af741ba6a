// mcrt_mixed.cu -- mixed-precision transport build.
//
// The transport and peel-off kernels of mcrt_sched.cuh / mcrt_peel.cuh
// compiled with MCRT_MIXED: scattering (rejection sampling, frame rotations,
// the peel-off phase matrix) runs in FP32.  The walk's geometry stays FP64,
// because testgrid resolves 1e-4 of a cell and the rim and equatorial cells
// are 6.5e-4 wide in cos(theta), beyond FP32 positions; the mixed walk drops
// the divisions instead (grid tests as products, one reciprocal per face
// quadratic, FMA contraction on).  Positions, face roots, the cumulative
// optical depth and its comparison with the sampled tau, opacities and all
// tallies are FP64.  The device code is
// compiled into its own namespace so that it can coexist with the FP64
// build's kernels; the launch parameters have the same layout.
#include <cuda_runtime.h>

#define MCRT_MIXED 1
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
