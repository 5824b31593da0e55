// FP64 raymarch kernels over FP32 or FP64 primitive pools (1, 4 and 32 frequency slots).
#include "march_impl.cuh"

namespace phx {
template cudaError_t launch_march<Mode::kFP64, float>(const MarchArgs<double, float>&, int, int, cudaStream_t,
                                                      LaunchShape*);
template cudaError_t launch_march<Mode::kFP64, double>(const MarchArgs<double, double>&, int, int, cudaStream_t,
                                                       LaunchShape*);
}  // namespace phx
