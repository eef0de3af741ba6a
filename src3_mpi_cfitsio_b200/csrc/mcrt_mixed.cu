// mcrt_mixed.cu -- mixed-precision transport build (FP32 walk and scattering,
// FP64 radial roots, optical-depth sums and tallies).
#include <cuda_runtime.h>

#include "mcrt_device.cuh"

namespace mcrt {

cudaError_t launch_transport_mixed(const LaunchParams&, int, cudaStream_t) { return cudaErrorNotSupported; }
int transport_mixed_blocks_per_sm() { return 1; }

}  // namespace mcrt
