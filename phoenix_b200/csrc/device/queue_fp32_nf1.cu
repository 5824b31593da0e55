// FP32 queue kernels, one frequency slot (register-cap variants 1, 3, 4 blocks/SM).
#include "queue_impl.cuh"

namespace phx {
template cudaError_t launch_queue_nf<Mode::kFP32, float, 1>(const QueueArgs<float, float>&, int, QueueShape, long long,
                                                            cudaStream_t, LaunchShape*);
template cudaError_t launch_ray_setup<Mode::kFP32, float>(const ItemDesc<float, float>&, long long, int, RayStart*,
                                                          cudaStream_t);
}  // namespace phx
