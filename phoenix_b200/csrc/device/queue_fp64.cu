// FP64 queue kernels (FP64 or FP32 primitives), one and four frequency slots.
#include "queue_impl.cuh"

namespace phx {
template cudaError_t launch_queue_nf<Mode::kFP64, double, 1>(const QueueArgs<double, double>&, int, QueueShape,
                                                             long long, cudaStream_t, LaunchShape*);
template cudaError_t launch_queue_nf<Mode::kFP64, double, 4>(const QueueArgs<double, double>&, int, QueueShape,
                                                             long long, cudaStream_t, LaunchShape*);
template cudaError_t launch_queue_nf<Mode::kFP64, float, 1>(const QueueArgs<double, float>&, int, QueueShape,
                                                            long long, cudaStream_t, LaunchShape*);
template cudaError_t launch_queue_nf<Mode::kFP64, float, 4>(const QueueArgs<double, float>&, int, QueueShape,
                                                            long long, cudaStream_t, LaunchShape*);
template cudaError_t launch_ray_setup<Mode::kFP64, double>(const ItemDesc<double, double>&, long long, int, RayStart*,
                                                           cudaStream_t);
template cudaError_t launch_ray_setup<Mode::kFP64, float>(const ItemDesc<double, float>&, long long, int, RayStart*,
                                                          cudaStream_t);
}  // namespace phx
