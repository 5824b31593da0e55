// Launch logic of the raymarch kernel (see march.cuh); each march_<mode>.cu instantiates it for one mode.
#pragma once

#include "march.cuh"

namespace phx {

namespace {

constexpr int kBlock = 128;

template <Mode M, class PT, int NF>
cudaError_t launch_nf(const MarchArgs<typename Policy<M>::R, PT>& args, int sms, int blocks_per_sm,
                      cudaStream_t stream, LaunchShape* shape) {
  auto kern = k_march<M, PT, NF, kBlock, 1>;
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, kern);
  if (e != cudaSuccess) return e;
  int bpsm = blocks_per_sm;
  if (bpsm <= 0) {
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bpsm, kern, kBlock, 0);
    if (e != cudaSuccess) return e;
    if (bpsm < 1) bpsm = 1;
  }
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
  kern<<<(unsigned)grid, kBlock, 0, stream>>>(args);
  return cudaGetLastError();
}

}  // namespace

template <Mode M, class PT>
cudaError_t launch_march(const MarchArgs<typename Policy<M>::R, PT>& args, int sms, int blocks_per_sm,
                         cudaStream_t stream, LaunchShape* shape) {
  const int nf = args.rc.nfreqs;
  if (nf <= 1) return launch_nf<M, PT, 1>(args, sms, blocks_per_sm, stream, shape);
  if (nf <= 4) return launch_nf<M, PT, 4>(args, sms, blocks_per_sm, stream, shape);
  return launch_nf<M, PT, kMaxFreqs>(args, sms, blocks_per_sm, stream, shape);
}

}  // namespace phx
