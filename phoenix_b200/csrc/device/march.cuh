// The fused raymarch kernel: a persistent grid of warps, one ray per lane, fed from a device job queue.
//
// Every pass of the march loop is one Ray::advance() per live lane (geodesic step + leaf lookups + the plasma
// stage of the sample + its transfer operator for every frequency).  A warp collects its finished lanes with a
// ballot, takes that many pixel jobs from the queue with one atomic and starts the new rays in those lanes
// (prefix-popcount ranks): when `refill_lanes` of its lanes have finished (checked every 64 passes; by default all
// 32) or at the end of a `period` of passes.  The reference kernel (src/device/kernel.cu:56-100) runs each pixel's
// whole inner loop in its lane and takes jobs with one atomic per warp; here the loop is resumable pass by pass, so
// the refill policy is a choice (refill_lanes, period), discussed beside kDefaultPeriod below: refilling single lanes
// as early as possible measured slowest.
//
// Device buffers a launch touches: the snapshot pool and job list (read), the FreqOut image (written once per
// pixel), optional per-pixel statistics, and a 16-word counter block (queue head + diagnostic sums).
#pragma once

#include <cuda_runtime.h>

#include "../core/ray.cuh"

namespace phx {

enum CounterSlot {
  kCtrQueue = 0,
  kCtrSteps = 1,
  kCtrPlasma = 2,
  kCtrBad = 3,
  kCtrScans = 4,
  kCtrFp64Steps = 5,
  kCtrFp64Ops = 6,
  kCtrRays = 7,
  kNumCounters = 16
};

template <class R, class PT>
struct MarchArgs {
  SnapView<R, PT> snap;
  SnapView<double, PT> snap_d;  // FP64 leaf geometry and constants (the mixed mode's geodesic)
  RenderConsts<R> rc;
  const int32_t* jobs;
  int64_t njobs;
  double* out;
  int32_t* pixstats;
  unsigned long long* counters;
  int32_t period;
  int32_t refill_lanes;  // finished lanes at which a warp refills before its period ends (checked every 64 passes)
};

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <Mode M, class PT, int NF, int kBlock, int kMinBlocks>
__global__ void __launch_bounds__(kBlock, kMinBlocks)
    k_march(const __grid_constant__ MarchArgs<typename Policy<M>::R, PT> A) {
  using RayT = Ray<M, PT, NF>;
  const unsigned lane = threadIdx.x & 31u;
  RayT ray;
  RayCounters ctr{};
  // per-lane sums in 32 bits (a launch gives a lane at most ~2^31 / lanes rays of <= max_steps steps: far below 2^32)
  unsigned steps = 0, nplasma = 0, bad = 0, rays = 0;
  bool live = false, drained = false;
  for (;;) {
    if (!drained) {
      const unsigned idle = __ballot_sync(0xffffffffu, !live);
      if (idle) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(&A.counters[kCtrQueue], (unsigned long long)__popc(idle));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= (unsigned long long)A.njobs) drained = true;
        if (!live) {
          const unsigned long long job = base + __popc(idle & ((1u << lane) - 1u));
          if (job < (unsigned long long)A.njobs) {
            const int32_t pix = A.jobs[job];
            // a job outside the image is skipped, never written (the host checks job lists it uploads itself)
            if (pix >= 0 && pix < A.rc.W * A.rc.H) {
              ray.init(A.snap, A.snap_d, A.rc, pix);
              live = true;
            }
          }
        }
      }
    }
    if (!__any_sync(0xffffffffu, live)) break;
    for (int it = 0; it < A.period; it++) {
      if (live) {
        live = ray.advance(A.snap, A.snap_d, A.rc, ctr);
        if (!live) {
          ray.write(A.out, A.rc.nfreqs);
          if (A.pixstats) {
            int32_t* ps = A.pixstats + 3 * (size_t)ray.pix;
            ps[0] = ray.steps;
            ps[1] = ray.nplasma;
            ps[2] = ray.bad;
          }
          steps += (unsigned)ray.steps;
          nplasma += (unsigned)ray.nplasma;
          bad += (unsigned)ray.bad;
          rays++;
        }
      }
      // a warp with refill_lanes finished lanes refills at once instead of at the end of the period
      if ((it & 63) == 63 && __popc(__ballot_sync(0xffffffffu, !live)) >= A.refill_lanes) break;
    }
  }
  const unsigned long long wsteps = warp_sum_u64(steps), wnplasma = warp_sum_u64(nplasma), wbad = warp_sum_u64(bad),
                           wrays = warp_sum_u64(rays);
  const unsigned long long scans = warp_sum_u64(ctr.scans);
  const unsigned long long f64s = warp_sum_u64(ctr.fp64_steps);
  const unsigned long long f64o = warp_sum_u64(ctr.fp64_ops);
  if (lane == 0) {
    atomicAdd(&A.counters[kCtrSteps], wsteps);
    atomicAdd(&A.counters[kCtrPlasma], wnplasma);
    atomicAdd(&A.counters[kCtrBad], wbad);
    atomicAdd(&A.counters[kCtrRays], wrays);
    if (scans) atomicAdd(&A.counters[kCtrScans], scans);
    if (f64s) atomicAdd(&A.counters[kCtrFp64Steps], f64s);
    if (f64o) atomicAdd(&A.counters[kCtrFp64Ops], f64o);
  }
}

// Refill policy of the single-image kernel: a warp takes new jobs when all its lanes have finished (refill_lanes 32,
// checked every 64 passes), or at the end of a period, by default longer than any ray.  Measured on B200 (FP32,
// centre-first job lists; ms for the 3 x 512^2 bench images / one 1024^2 image of 3 frequencies): a refill of the
// finished lanes every 64 passes 247 / 480, every 256 243 / 433, every 4096 233 / 370; whole-warp refill 231 / 363;
// refill once 24 lanes have finished 237 / 378, 8 lanes 242 / 433.  Lanes refilled one or two at a time start their
// rays in a different phase than their neighbours (far from the hole, no plasma, long steps): the warp then pays
// for both phases' code at every pass, which costs more than the lanes a whole-warp refill leaves idle behind the
// warp's longest ray; rays that start together from neighbouring pixels stay in step.  The queue kernel (batches,
// serving) uses the same policy by default; batches autotune it.
constexpr int kDefaultPeriod = 1 << 20;
constexpr int kDefaultQueuePeriod = 1 << 20;

// Launch entry per (mode, prim type): picks the frequency-slot instantiation and the launch shape.
struct LaunchShape {
  int block, grid, regs, local_bytes, blocks_per_sm;
};

// One frequency-slot instantiation (defined in march_impl.cuh, instantiated by the march_*.cu files).
template <Mode M, class PT, int NF>
cudaError_t launch_nf(const MarchArgs<typename Policy<M>::R, PT>& args, int sms, int blocks_per_sm,
                      cudaStream_t stream, LaunchShape* shape);

template <Mode M, class PT>
cudaError_t launch_march(const MarchArgs<typename Policy<M>::R, PT>& args, int sms, int blocks_per_sm,
                         cudaStream_t stream, LaunchShape* shape);

}  // namespace phx
