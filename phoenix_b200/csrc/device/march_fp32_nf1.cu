// FP32 raymarch kernels, one frequency slot (register-cap variants 1, 3, 4 blocks/SM).
#include "march_impl.cuh"

namespace phx {
template cudaError_t launch_nf<Mode::kFP32, float, 1>(const MarchArgs<float, float>&, int, int, cudaStream_t,
                                                          LaunchShape*);
}  // namespace phx
