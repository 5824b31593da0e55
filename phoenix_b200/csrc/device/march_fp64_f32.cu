// FP64 raymarch kernels over an FP32 primitive pool.
#include "march_impl.cuh"

namespace phx {
template cudaError_t launch_nf<Mode::kFP64, float, 1>(const MarchArgs<double, float>&, int, int, cudaStream_t,
                                                          LaunchShape*);
template cudaError_t launch_nf<Mode::kFP64, float, 4>(const MarchArgs<double, float>&, int, int, cudaStream_t,
                                                          LaunchShape*);
template cudaError_t launch_nf<Mode::kFP64, float, 32>(const MarchArgs<double, float>&, int, int, cudaStream_t,
                                                          LaunchShape*);
}  // namespace phx
