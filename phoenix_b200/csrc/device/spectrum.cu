// Per-frequency image totals on the device: the reference's host::output::compute_spec and compute_tau
// (src/host/io/output.hpp:43-74) without downloading the image.
//
//   I, Q, U, V  summed over the pixels whose I+Q+U+V is finite, times the pixel solid angle and 1e23 (Jy);
//   tau, tauF   means over the pixels whose six values sum to a finite number (0 when there are none).
//
// One thread-block cluster of kSpecCluster CTAs per frequency: each CTA sums a strided share of the pixels into
// FP64 partials (warp shuffles, then its warps in a fixed order); CTA 0 of the cluster then reads the other CTAs'
// partials through distributed shared memory, in rank order, and writes the record.  The result is deterministic
// (no atomics) and nothing beyond the image and the output records is touched.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cmath>
#include <stdexcept>

#include "../host/render_setup.hpp"
#include "internal.hpp"

namespace cg = cooperative_groups;
using namespace phx_capi;

namespace {

constexpr int kSpecCluster = 8;
constexpr int kSpecThreads = 512;
constexpr int kSpecWarps = kSpecThreads / 32;

struct SpecPart {
  double s[6];              // I, Q, U, V, tau, tauF
  unsigned long long n[2];  // pixels in the flux sum, in the optical-depth means
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ unsigned long long warp_sum(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

__global__ void __cluster_dims__(kSpecCluster, 1, 1) __launch_bounds__(kSpecThreads)
    k_spectrum(const double2* __restrict__ res, long long npix, int nfreqs, double jy_per_unit,
               PhxSpectrum* __restrict__ out) {
  __shared__ SpecPart warp_part[kSpecWarps];
  __shared__ SpecPart cta_part;
  cg::cluster_group cluster = cg::this_cluster();
  const unsigned rank = cluster.block_rank();
  const int f = blockIdx.y;
  double s[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  unsigned long long nflux = 0, ntau = 0;
  const long long stride = (long long)kSpecCluster * kSpecThreads;
  for (long long p = (long long)rank * kSpecThreads + threadIdx.x; p < npix; p += stride) {
    const double2* r = res + ((size_t)p * nfreqs + f) * 3;  // one 48-byte record: three 16-byte loads
    const double2 iq = __ldg(r), uv = __ldg(r + 1), tt = __ldg(r + 2);
    const double stokes = iq.x + iq.y + uv.x + uv.y;
    if (isfinite(stokes)) {
      s[0] += iq.x;
      s[1] += iq.y;
      s[2] += uv.x;
      s[3] += uv.y;
      nflux++;
    }
    if (isfinite(stokes + tt.x + tt.y)) {
      s[4] += tt.x;
      s[5] += tt.y;
      ntau++;
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 6; q++) s[q] = warp_sum(s[q]);
  nflux = warp_sum(nflux);
  ntau = warp_sum(ntau);
  if (lane == 0) {
#pragma unroll
    for (int q = 0; q < 6; q++) warp_part[warp].s[q] = s[q];
    warp_part[warp].n[0] = nflux;
    warp_part[warp].n[1] = ntau;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    SpecPart t = warp_part[0];
    for (int w = 1; w < kSpecWarps; w++) {
      for (int q = 0; q < 6; q++) t.s[q] += warp_part[w].s[q];
      t.n[0] += warp_part[w].n[0];
      t.n[1] += warp_part[w].n[1];
    }
    cta_part = t;
  }
  cluster.sync();  // every CTA's partial is in its shared memory
  if (rank == 0 && threadIdx.x == 0) {
    SpecPart t = cta_part;
    for (unsigned c = 1; c < kSpecCluster; c++) {
      const SpecPart* o = cluster.map_shared_rank(&cta_part, c);
      for (int q = 0; q < 6; q++) t.s[q] += o->s[q];
      t.n[0] += o->n[0];
      t.n[1] += o->n[1];
    }
    PhxSpectrum rec;
    for (int q = 0; q < 4; q++) rec.IQUV[q] = t.s[q] * jy_per_unit;
    rec.tau_mean = t.n[1] ? t.s[4] / (double)t.n[1] : 0.0;
    rec.tauF_mean = t.n[1] ? t.s[5] / (double)t.n[1] : 0.0;
    rec.n_flux = (int64_t)t.n[0];
    rec.n_tau = (int64_t)t.n[1];
    out[f] = rec;
  }
  cluster.sync();  // CTA 0 has read the others' shared memory before they exit
}

}  // namespace

namespace phx_capi {

void launch_spectrum(const PhxRenderParams& p, const PhxFreqOut* d_res, PhxSpectrum* d_spec, cudaStream_t st) {
  if ((reinterpret_cast<uintptr_t>(d_res) & 15u) != 0) throw std::invalid_argument("d_res must be 16-byte aligned");
  const long long npix = (long long)p.img_width * p.img_height;
  const double jy = phx::pixel_solid_angle(p) * phx::cgs::jansky;
  const dim3 grid(kSpecCluster, p.nfreqs), block(kSpecThreads);
  k_spectrum<<<grid, block, 0, st>>>(reinterpret_cast<const double2*>(d_res), npix, p.nfreqs, jy, d_spec);
  ck(cudaGetLastError(), "spectrum launch");
}

}  // namespace phx_capi

extern "C" int phx_spectrum_async(const PhxRenderParams* p, const PhxFreqOut* d_res, PhxSpectrum* d_spec,
                                  void* stream) {
  return guarded([&]() -> int {
    if (!p || !d_res || !d_spec) throw std::invalid_argument("null argument");
    phx::check_params(*p);
    launch_spectrum(*p, d_res, d_spec, (cudaStream_t)stream);
    return PHX_OK;
  });
}
