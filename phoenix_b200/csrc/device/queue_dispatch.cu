// Frequency-slot dispatch of the queue kernels and the queue reset kernel.
#include "queue.cuh"

namespace phx {

template <Mode M, class PT, int NF>
cudaError_t launch_queue_nf(const QueueArgs<typename Policy<M>::R, PT>& args, int sms, QueueShape q,
                            long long max_rays, cudaStream_t stream, LaunchShape* shape);

template <Mode M, class PT>
cudaError_t launch_queue(const QueueArgs<typename Policy<M>::R, PT>& args, int nf_slots, int sms, QueueShape q,
                         long long max_rays, cudaStream_t stream, LaunchShape* shape) {
  if (nf_slots <= 1) return launch_queue_nf<M, PT, 1>(args, sms, q, max_rays, stream, shape);
  if (nf_slots <= 4) return launch_queue_nf<M, PT, 4>(args, sms, q, max_rays, stream, shape);
  if constexpr (M == Mode::kFP32) return launch_queue_nf<M, PT, kMaxFreqs>(args, sms, q, max_rays, stream, shape);
  return cudaErrorInvalidValue;  // more than 4 frequencies per image: FP32 only
}

template cudaError_t launch_queue<Mode::kFP32, float>(const QueueArgs<float, float>&, int, int, QueueShape, long long,
                                                      cudaStream_t, LaunchShape*);
template cudaError_t launch_queue<Mode::kMixed, float>(const QueueArgs<float, float>&, int, int, QueueShape, long long,
                                                       cudaStream_t, LaunchShape*);
template cudaError_t launch_queue<Mode::kFP64, float>(const QueueArgs<double, float>&, int, int, QueueShape, long long,
                                                      cudaStream_t, LaunchShape*);
template cudaError_t launch_queue<Mode::kFP64, double>(const QueueArgs<double, double>&, int, int, QueueShape,
                                                       long long, cudaStream_t, LaunchShape*);

__global__ void k_queue_reset(unsigned long long* ctl, unsigned long long* counters, unsigned long long* item_ctr,
                              long long n_item_words, unsigned long long ntiles) {
  const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  if (tid < kQWords) ctl[tid] = tid == kQTail ? ntiles : 0ull;
  if (tid < kNumCounters) counters[tid] = 0ull;
  for (long long i = tid; i < n_item_words; i += stride) item_ctr[i] = 0ull;
}

cudaError_t launch_queue_reset(unsigned long long* ctl, unsigned long long* counters, unsigned long long* item_ctr,
                               long long n_item_words, unsigned long long ntiles, cudaStream_t stream) {
  long long blocks = (n_item_words + 255) / 256;
  if (blocks < 1) blocks = 1;
  if (blocks > 1024) blocks = 1024;
  k_queue_reset<<<(unsigned)blocks, 256, 0, stream>>>(ctl, counters, item_ctr, n_item_words, ntiles);
  return cudaGetLastError();
}

}  // namespace phx
