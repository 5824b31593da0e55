// Launch logic of the raymarch kernel (see march.cuh); each march_<mode>_nf<slots>.cu file instantiates launch_nf.
#pragma once

#include "march.cuh"

namespace phx {

// Launch shapes.  `blocks_per_sm` names a register-cap variant by its resident warps per SM / 4:
//   1: 128-thread blocks, up to 255 registers (the compiler takes 192 in FP32: 2 blocks, 8 warps per SM);
//   3: 168 registers, 12 warps per SM;   4: 128 registers, 16 warps per SM.
// Variants 3 and 4 run as ONE block of 384 / 512 threads per SM when the job list gives every SM such a block, and as
// 3 / 4 blocks of 128 threads otherwise (small images then still spread over all SMs).  On B200 the whole-SM block
// measured faster than the same warps in 128-thread blocks: FP32, 3 x 512^2 bench images, 16 warps 326 ms as one
// block vs 379 ms as four; 12 warps 336 vs 349 ms.
template <Mode M, class PT, int NF, int kBlock, int kMinBlocks>
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

// Default variant per mode (measured on B200, 3 x 512^2 bench images): FP32 4 (128 registers, 16 warps); mixed with one
// frequency slot 4 (128 registers, 140 bytes of spills: 474 ms vs 484 ms at 168 registers, 12 warps), mixed with more
// slots 3 (4% faster than uncapped in 128-thread blocks); FP64 uncapped.
template <Mode M, int NF>
constexpr int default_blocks_per_sm() {
  return M == Mode::kFP32 ? 4 : M == Mode::kMixed ? (NF == 1 ? 4 : 3) : 1;
}

// The variant for `blocks_per_sm` (0 = the mode's default).  FP64 and the 32-slot kernels are compiled uncapped only;
// mixed offers 1 and 3, and 4 with one frequency slot.
template <Mode M, class PT, int NF>
cudaError_t launch_nf(const MarchArgs<typename Policy<M>::R, PT>& args, int sms, int blocks_per_sm,
                      cudaStream_t stream, LaunchShape* shape) {
  if constexpr (M == Mode::kFP64 || NF > 4) {
    (void)blocks_per_sm;
    return launch_mb<M, PT, NF, 128, 1>(args, sms, stream, shape);
  } else {
    const int bps = blocks_per_sm > 0 ? blocks_per_sm : default_blocks_per_sm<M, NF>();
    const bool whole = args.njobs >= (long long)sms * 128 * bps;  // a whole-SM block for every SM
    if (bps == 3) {
      return whole ? launch_mb<M, PT, NF, 384, 1>(args, sms, stream, shape)
                   : launch_mb<M, PT, NF, 128, 3>(args, sms, stream, shape);
    }
    if constexpr (M == Mode::kFP32 || (M == Mode::kMixed && NF == 1)) {
      if (bps == 4) {
        return whole ? launch_mb<M, PT, NF, 512, 1>(args, sms, stream, shape)
                     : launch_mb<M, PT, NF, 128, 4>(args, sms, stream, shape);
      }
    }
    return launch_mb<M, PT, NF, 128, 1>(args, sms, stream, shape);
  }
}

}  // namespace phx
