// Launch logic of the queue kernel (see queue.cuh); each queue_*.cu file instantiates launch_queue_nf.
#pragma once

#include <algorithm>

#include "queue.cuh"

namespace phx {

constexpr int kQueueBlock = 128;

template <Mode M, class PT, int NF, int kMinBlocks>
cudaError_t launch_queue_mb(const QueueArgs<typename Policy<M>::R, PT>& args, int sms, int period, long long max_rays,
                            cudaStream_t stream, LaunchShape* shape) {
  auto kern = k_queue<M, PT, NF, kQueueBlock, kMinBlocks>;
  // the rays' transfer records (shared-memory kernels; 0 otherwise)
  const size_t smem = Ray<M, PT, NF>::kSmemPerThread * kQueueBlock;
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, kern);
  if (e != cudaSuccess) return e;
  if (smem > 48 * 1024) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  int bpsm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bpsm, kern, kQueueBlock, smem);
  if (e != cudaSuccess) return e;
  if (bpsm < 1) bpsm = 1;
  long long grid = (long long)bpsm * sms;
  if (max_rays > 0) grid = std::min(grid, (max_rays + kQueueBlock - 1) / kQueueBlock);
  if (grid < 1) grid = 1;
  shape->block = kQueueBlock;
  shape->grid = (int)grid;
  shape->regs = fa.numRegs;
  shape->local_bytes = (int)fa.localSizeBytes;
  shape->blocks_per_sm = bpsm;
  QueueArgs<typename Policy<M>::R, PT> a = args;
  a.period = period > 0 ? period : 32;
  kern<<<(unsigned)grid, kQueueBlock, smem, stream>>>(a);
  return cudaGetLastError();
}

// Register-cap variants as for the single-image kernel: FP32 is compiled for 1, 3 and 4 resident 128-thread blocks
// per SM with one and four frequency slots; mixed for 1 and 3; FP64 and 32 slots uncapped.
template <Mode M, class PT, int NF>
cudaError_t launch_queue_nf(const QueueArgs<typename Policy<M>::R, PT>& args, int sms, QueueShape q,
                            long long max_rays, cudaStream_t stream, LaunchShape* shape) {
  if constexpr (M == Mode::kFP64 || NF > 4) {
    return launch_queue_mb<M, PT, NF, 1>(args, sms, q.period, max_rays, stream, shape);
  } else if constexpr (M == Mode::kMixed) {
    if (q.blocks_per_sm == 3) return launch_queue_mb<M, PT, NF, 3>(args, sms, q.period, max_rays, stream, shape);
    return launch_queue_mb<M, PT, NF, 1>(args, sms, q.period, max_rays, stream, shape);
  } else {
    switch (q.blocks_per_sm) {
      case 1:
      case 2:
        return launch_queue_mb<M, PT, NF, 1>(args, sms, q.period, max_rays, stream, shape);
      case 4:
        return launch_queue_mb<M, PT, NF, 4>(args, sms, q.period, max_rays, stream, shape);
      default:
        return launch_queue_mb<M, PT, NF, 3>(args, sms, q.period, max_rays, stream, shape);
    }
  }
}

}  // namespace phx
