// FP32 queue kernels, four frequency slots (register-cap variants 1, 3, 4 blocks/SM) and 32 slots (uncapped).
#include "queue_impl.cuh"

namespace phx {
template cudaError_t launch_queue_nf<Mode::kFP32, float, 4>(const QueueArgs<float, float>&, int, QueueShape, long long,
                                                            cudaStream_t, LaunchShape*);
template cudaError_t launch_queue_nf<Mode::kFP32, float, kMaxFreqs>(const QueueArgs<float, float>&, int, QueueShape,
                                                                    long long, cudaStream_t, LaunchShape*);
}  // namespace phx
