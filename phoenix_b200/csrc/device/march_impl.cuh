// Launch logic of the raymarch kernel (see march.cuh); each march_<mode>_nf<slots>.cu file instantiates launch_nf.
#pragma once

#include "march.cuh"

namespace phx {

constexpr int kBlock = 128;

template <Mode M, class PT, int NF, int kMinBlocks>
cudaError_t launch_mb(const MarchArgs<typename Policy<M>::R, PT>& args, int sms, cudaStream_t stream,
                      LaunchShape* shape) {
  auto kern = k_march<M, PT, NF, kBlock, kMinBlocks>;
  // the rays' transfer records (shared-memory kernels; 0 otherwise)
  const size_t smem = Ray<M, PT, NF>::kSmemPerThread * kBlock;
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, kern);
  if (e != cudaSuccess) return e;
  if (smem > 48 * 1024) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  int bpsm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bpsm, kern, kBlock, smem);
  if (e != cudaSuccess) return e;
  if (bpsm < 1) bpsm = 1;
  long long grid = (long long)bpsm * sms;
  const long long need = (args.njobs + kBlock - 1) / kBlock;
  if (grid > need) grid = need;
  if (grid < 1) grid = 1;
  shape->block = kBlock;
  shape->grid = (int)grid;
  shape->regs = fa.numRegs;
  shape->local_bytes = (int)fa.localSizeBytes;
  shape->blocks_per_sm = bpsm;
  if (args.njobs <= 0) return cudaSuccess;
  kern<<<(unsigned)grid, kBlock, smem, stream>>>(args);
  return cudaGetLastError();
}

// Register-cap variants: `blocks_per_sm` picks the instantiation compiled for that many resident 128-thread blocks
// per SM (__launch_bounds__ min blocks: 1 -> up to 255 registers, 3 -> 168, 4 -> 128; 0 = default).  FP64 and the 32-slot
// variants are compiled uncapped only.
template <Mode M, class PT, int NF>
cudaError_t launch_nf(const MarchArgs<typename Policy<M>::R, PT>& args, int sms, int blocks_per_sm,
                      cudaStream_t stream, LaunchShape* shape) {
  if constexpr (M == Mode::kFP64 || NF > 4) {
    (void)blocks_per_sm;
    return launch_mb<M, PT, NF, 1>(args, sms, stream, shape);
  } else {
    switch (blocks_per_sm) {
      case 1:
      case 2:
        return launch_mb<M, PT, NF, 1>(args, sms, stream, shape);
      case 3:
        return launch_mb<M, PT, NF, 3>(args, sms, stream, shape);
      case 4:
        return launch_mb<M, PT, NF, 4>(args, sms, stream, shape);
      default:  // measured on B200: FP32 3 resident blocks (168 registers); mixed uncapped (it spills at 168)
        if constexpr (M == Mode::kMixed) return launch_mb<M, PT, NF, 1>(args, sms, stream, shape);
        else return launch_mb<M, PT, NF, 3>(args, sms, stream, shape);
    }
  }
}

}  // namespace phx
