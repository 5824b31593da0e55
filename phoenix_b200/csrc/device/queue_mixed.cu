// Mixed-precision queue kernels, one and four frequency slots.
#include "queue_impl.cuh"

namespace phx {
template cudaError_t launch_queue_nf<Mode::kMixed, float, 1>(const QueueArgs<float, float>&, int, QueueShape, long long,
                                                             cudaStream_t, LaunchShape*);
template cudaError_t launch_queue_nf<Mode::kMixed, float, 4>(const QueueArgs<float, float>&, int, QueueShape, long long,
                                                             cudaStream_t, LaunchShape*);
template cudaError_t launch_ray_setup<Mode::kMixed, float>(const ItemDesc<float, float>&, long long, int, RayStart*,
                                                           cudaStream_t);
}  // namespace phx
