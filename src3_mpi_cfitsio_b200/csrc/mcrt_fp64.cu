// mcrt_fp64.cu -- FP64 transport build.  Compiled with --fmad=false so that
// every FP64 add/multiply is a separate IEEE operation, as in the oracle.
#include <cuda_runtime.h>

#include <algorithm>

#include "mcrt_sched.cuh"
#include "mcrt_peel.cuh"
#include "mcrt_wave.cuh"
#include "mcrt_batch.cuh"
#include "mcrt_setemiss.cuh"

namespace mcrt {

static_assert(sizeof(LaunchParams) % 4 == 0, "LaunchParams is copied as 32-bit words");

cudaError_t launch_batch_fp64(const LaunchParams* params, const BatchItem* items, int64_t nitems,
                              unsigned long long* item_next, unsigned long long* chunk_next, int32_t event_batch,
                              int grid, cudaStream_t s) {
  transport_batch<<<grid, kBlock, 0, s>>>(params, items, nitems, item_next, chunk_next, event_batch);
  return cudaGetLastError();
}

int batch_fp64_blocks_per_sm() {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, transport_batch, kBlock, 0) != cudaSuccess) return 1;
  return n > 0 ? n : 1;
}

cudaError_t launch_setemiss(const SetemissArgs& a, double* tmp, cudaStream_t s) {
  const dim3 grid((unsigned)a.nT, (unsigned)a.nopac);
  setemiss_tables<<<grid, kSetemissBlock, (size_t)2 * a.nnu * sizeof(double), s>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || a.ndg >= a.nopac) return e;
  const int ngas = a.nopac - a.ndg;
  setemiss_smooth<<<(ngas + 63) / 64, 64, 0, s>>>(a.kappap, tmp, a.nT, a.ndg, a.nopac);
  return cudaGetLastError();
}

cudaError_t launch_wave_init(const WaveArgs& w, cudaStream_t s) {
  const int grid = (int)std::min<int64_t>((w.slots + 255) / 256, 4096);
  wave_init<<<grid > 0 ? grid : 1, 256, 0, s>>>(w);
  return cudaGetLastError();
}

cudaError_t launch_wave_event_fp64(const LaunchParams& p, const WaveArgs& w, int grid, cudaStream_t s) {
  wave_event<<<grid, kBlock, 0, s>>>(p, w);
  return cudaGetLastError();
}

cudaError_t launch_wave_walk_fp64(const LaunchParams& p, const WaveArgs& w, int grid, cudaStream_t s) {
  wave_walk<<<grid, kBlock, 0, s>>>(p, w);
  return cudaGetLastError();
}

cudaError_t launch_wave_tail_fp64(const LaunchParams& p, const WaveArgs& w, int grid, cudaStream_t s) {
  wave_tail<<<grid, kBlock, 0, s>>>(p, w);
  return cudaGetLastError();
}

int wave_tail_fp64_blocks_per_sm() {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, wave_tail, kBlock, 0) != cudaSuccess) return 1;
  return n > 0 ? n : 1;
}

int wave_event_fp64_blocks_per_sm() {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, wave_event, kBlock, 0) != cudaSuccess) return 1;
  return n > 0 ? n : 1;
}

int wave_walk_fp64_blocks_per_sm() {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, wave_walk, kBlock, 0) != cudaSuccess) return 1;
  return n > 0 ? n : 1;
}

cudaError_t launch_transport_fp64(const LaunchParams& p, int grid, cudaStream_t s) {
  transport_fp64<<<grid, kBlock, 0, s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_transport_sched_fp64(const LaunchParams& p, int grid, cudaStream_t s) {
  transport_sched<<<grid, kBlock, 0, s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_peel_fp64(const LaunchParams& p, unsigned long long* next_item, int grid, cudaStream_t s) {
  peel_sched<<<grid, kBlock, 0, s>>>(p, next_item);
  return cudaGetLastError();
}

int peel_fp64_blocks_per_sm() {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, peel_sched, kBlock, 0) != cudaSuccess) return 1;
  return n > 0 ? n : 1;
}

int transport_sched_fp64_blocks_per_sm() {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, transport_sched, kBlock, 0) != cudaSuccess) return 1;
  return n > 0 ? n : 1;
}

cudaError_t launch_diffusion_finalize(const DevModel& m, const int32_t* ndiff, const double* tdust0, double* tdust,
                                      double nphot, cudaStream_t s) {
  diffusion_finalize<<<256, 256, 0, s>>>(m, ndiff, tdust0, tdust, nphot);
  return cudaGetLastError();
}

int transport_fp64_blocks_per_sm() {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, transport_fp64, kBlock, 0) != cudaSuccess) return 1;
  return n > 0 ? n : 1;
}

}  // namespace mcrt
