// FP32 raymarch kernels, 4 and 32 frequency slots.
#include "march_impl.cuh"

namespace phx {
template cudaError_t launch_nf<Mode::kFP32, float, 4>(const MarchArgs<float, float>&, int, int, cudaStream_t,
                                                          LaunchShape*);
template cudaError_t launch_nf<Mode::kFP32, float, 32>(const MarchArgs<float, float>&, int, int, cudaStream_t,
                                                          LaunchShape*);
}  // namespace phx
