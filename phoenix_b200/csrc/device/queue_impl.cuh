// Launch logic of the queue kernel (see queue.cuh); each queue_*.cu file instantiates launch_queue_nf.
#pragma once

#include <algorithm>

#include "queue.cuh"

namespace phx {

template <Mode M, class PT, int NF, int kQueueBlock, int kMinBlocks>
cudaError_t launch_queue_mb(const QueueArgs<typename Policy<M>::R, PT>& args, int sms, QueueShape qs, long long max_rays,
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
  a.period = qs.period > 0 ? qs.period : 32;
  a.refill_lanes = qs.refill_lanes > 0 ? qs.refill_lanes : 32;
  kern<<<(unsigned)grid, kQueueBlock, smem, stream>>>(a);
  return cudaGetLastError();
}

// Register-cap variants and block shapes as for the single-image kernel (march_impl.cuh): `blocks_per_sm` 1 -> 128-thread
// blocks at up to 255 registers; 3 / 4 -> 168 / 128 registers as one 384 / 512-thread block per SM, or as 128-thread
// blocks when the work (max_rays; <= 0: unbounded, a serving loop) cannot give every SM a whole block.  FP32 offers
// 1, 3, 4; mixed 1 and 3, and 4 with one frequency slot; FP64 and 32 slots are uncapped only.
template <Mode M, class PT, int NF>
cudaError_t launch_queue_nf(const QueueArgs<typename Policy<M>::R, PT>& args, int sms, QueueShape q,
                            long long max_rays, cudaStream_t stream, LaunchShape* shape) {
  if constexpr (M == Mode::kFP64 || NF > 4) {
    return launch_queue_mb<M, PT, NF, 128, 1>(args, sms, q, max_rays, stream, shape);
  } else {
    const int bps = q.blocks_per_sm > 0 ? q.blocks_per_sm : default_queue_blocks_per_sm<M, NF>();
    const bool whole = max_rays <= 0 || max_rays >= (long long)sms * 128 * bps;
    if (bps == 3) {
      return whole ? launch_queue_mb<M, PT, NF, 384, 1>(args, sms, q, max_rays, stream, shape)
                   : launch_queue_mb<M, PT, NF, 128, 3>(args, sms, q, max_rays, stream, shape);
    }
    if constexpr (M == Mode::kFP32 || (M == Mode::kMixed && NF == 1)) {
      if (bps == 4) {
        return whole ? launch_queue_mb<M, PT, NF, 512, 1>(args, sms, q, max_rays, stream, shape)
                     : launch_queue_mb<M, PT, NF, 128, 4>(args, sms, q, max_rays, stream, shape);
      }
    }
    return launch_queue_mb<M, PT, NF, 128, 1>(args, sms, q, max_rays, stream, shape);
  }
}

template <Mode M, class PT>
cudaError_t launch_ray_setup(const ItemDesc<typename Policy<M>::R, PT>& item, long long njobs, int sms,
                             RayStart* out, cudaStream_t stream) {
  using R = typename Policy<M>::R;
  using G = typename Policy<M>::G;
  if (njobs <= 0) return cudaSuccess;
  const long long blocks = std::min<long long>((njobs + 127) / 128, (long long)sms * 16);
  const G a = sizeof(G) == sizeof(R) ? G(item.snap.a) : G(item.snap_d.a);
  const G hs = sizeof(G) == sizeof(R) ? G(item.snap.hs) : G(item.snap_d.hs);
  k_ray_setup<G, R><<<(unsigned)blocks, 128, 0, stream>>>(item.rc, a, hs, item.jobs, njobs, out);
  return cudaGetLastError();
}

}  // namespace phx
