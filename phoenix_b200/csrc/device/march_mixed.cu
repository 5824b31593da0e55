// Mixed-precision raymarch kernels (1, 4 and 32 frequency slots).
#include "march_impl.cuh"

namespace phx {
template cudaError_t launch_march<Mode::kMixed, float>(const MarchArgs<float, float>&, int, int, cudaStream_t,
                                                       LaunchShape*);
}  // namespace phx
