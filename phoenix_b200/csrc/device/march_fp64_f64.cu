// FP64 raymarch kernels over an FP64 primitive pool.
#include "march_impl.cuh"

namespace phx {
template cudaError_t launch_nf<Mode::kFP64, double, 1>(const MarchArgs<double, double>&, int, int, cudaStream_t,
                                                          LaunchShape*);
template cudaError_t launch_nf<Mode::kFP64, double, 4>(const MarchArgs<double, double>&, int, int, cudaStream_t,
                                                          LaunchShape*);
template cudaError_t launch_nf<Mode::kFP64, double, 32>(const MarchArgs<double, double>&, int, int, cudaStream_t,
                                                          LaunchShape*);
}  // namespace phx
