// Frequency-slot dispatch of the raymarch kernels (the instantiations live in the march_*_nf*.cu files).
#include "march.cuh"

namespace phx {

template <Mode M, class PT>
cudaError_t launch_march(const MarchArgs<typename Policy<M>::R, PT>& args, int sms, int blocks_per_sm,
                         cudaStream_t stream, LaunchShape* shape) {
  const int nf = args.rc.nfreqs;
  if (nf <= 1) return launch_nf<M, PT, 1>(args, sms, blocks_per_sm, stream, shape);
  if (nf <= 4) return launch_nf<M, PT, 4>(args, sms, blocks_per_sm, stream, shape);
  return launch_nf<M, PT, kMaxFreqs>(args, sms, blocks_per_sm, stream, shape);
}

template cudaError_t launch_march<Mode::kFP32, float>(const MarchArgs<float, float>&, int, int, cudaStream_t,
                                                      LaunchShape*);
template cudaError_t launch_march<Mode::kMixed, float>(const MarchArgs<float, float>&, int, int, cudaStream_t,
                                                       LaunchShape*);
template cudaError_t launch_march<Mode::kFP64, float>(const MarchArgs<double, float>&, int, int, cudaStream_t,
                                                      LaunchShape*);
template cudaError_t launch_march<Mode::kFP64, double>(const MarchArgs<double, double>&, int, int, cudaStream_t,
                                                       LaunchShape*);

}  // namespace phx
