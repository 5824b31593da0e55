// Mixed-precision raymarch kernels, one frequency slot (register-cap variants).
#include "march_impl.cuh"

namespace phx {
template cudaError_t launch_nf<Mode::kMixed, float, 1>(const MarchArgs<float, float>&, int, int, cudaStream_t,
                                                          LaunchShape*);
}  // namespace phx
