// mcrt_fp64.cu -- FP64 transport build.  Compiled with --fmad=false so that
// every FP64 add/multiply is a separate IEEE operation, as in the oracle.
#include <cuda_runtime.h>

#include "mcrt_sched.cuh"
#include "mcrt_peel.cuh"

namespace mcrt {

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
