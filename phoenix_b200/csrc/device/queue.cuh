// The queue-fed raymarch kernel: many images (items) in one persistent launch.
//
// A batch or a stream of render requests is cut into ray tiles: tile t holds up to `tile_rays` consecutive jobs of
// one item (pixels of one image, in that image's job order).  Ray slot s belongs to tile s / tile_rays.  The tiles
// sit in a ring in device memory and a control block holds the queue head (ray slots claimed) and tail (tiles
// published).  Lanes claim slots with one atomic per warp, exactly as the single-image kernel claims jobs, so one
// warp may march rays of several images at once; each lane reads its image's constants and snapshot view from the
// item table in device memory instead of the kernel's parameter space.
//
// Batches publish every tile before the launch (the tail never moves): the kernel ends when the claims pass the
// tail.  A serving loop publishes tiles while the kernel runs: lanes whose claimed slot is not published yet keep
// the claim and retry at the next refill point; a warp with no live ray sleeps between polls and leaves when the host
// sets the stop word, or after `idle_limit` polls with the status word set (every wait in the kernel is bounded).
//
// Host-side rules that make the reads safe without cache maintenance:
//  * an item descriptor and its job list are written before the first tile that names the item is published, and are
//    not rewritten while a kernel that may have read them runs (descriptors are 128-byte aligned, so reading one
//    never caches a neighbour's bytes);
//  * tiles are read through L2 (ld.global.cg) because ring slots are reused; the tail is read with acquire order.
//
// When a ray ends its FreqOut records are written, then its item's counters are bumped; the lane that completes an
// item fences and raises the item's completion word (host-mapped memory for a serving loop).
#pragma once

#include <cuda_runtime.h>

#include "../core/ray.cuh"
#include "march.cuh"

namespace phx {

struct TileDesc {
  int32_t item;   // index into the item table
  int32_t first;  // first job of the tile in the item's job list
  int32_t count;  // jobs in the tile (<= tile_rays)
  int32_t pad;
};

enum ItemCounter {
  kItRays = 0,
  kItSteps = 1,
  kItPlasma = 2,
  kItBad = 3,
  kItemCounters = 8
};

enum QueueWord { kQHead = 0, kQTail = 1, kQStop = 2, kQStatus = 3, kQWords = 16 };

template <class R, class PT>
struct alignas(128) ItemDesc {
  RenderConsts<R> rc;
  SnapView<R, PT> snap;
  SnapView<double, PT> snap_d;   // FP64 leaf geometry and constants (the mixed mode's geodesic)
  const int32_t* jobs;
  const RayStart* starts;        // camera set-up of each job (k_ray_setup), or null: set up by the lane that takes it
  double* out;                   // FreqOut records of the image
  int32_t* pixstats;             // optional per-pixel (steps, segments, bad)
  unsigned long long* ctr;       // kItemCounters words
  unsigned long long nrays;      // jobs of the item over all its tiles
  volatile int32_t* done;        // completion word (0 -> 1), or null
};

template <class R, class PT>
struct QueueArgs {
  const ItemDesc<R, PT>* items;
  const TileDesc* tiles;
  unsigned long long* ctl;       // kQWords control words
  unsigned long long* counters;  // kernel-wide sums (the single-image kernel's counter block)
  unsigned tile_mask;            // ring capacity - 1 (a power of two)
  int32_t tile_rays;
  int32_t period;
  int32_t refill_lanes;          // finished lanes at which a warp claims new slots before its period ends
  int32_t idle_ns;               // sleep between polls of an idle warp; 0: leave once the published tiles are drained
  long long idle_limit;          // polls before an idle warp gives up (status word set)
};

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned long long ld_volatile_u64(const unsigned long long* p) {
  return *reinterpret_cast<const volatile unsigned long long*>(p);
}

constexpr unsigned long long kNoClaim = ~0ull;

template <Mode M, class PT, int NF, int kBlock, int kMinBlocks>
__global__ void __launch_bounds__(kBlock, kMinBlocks)
    k_queue(const __grid_constant__ QueueArgs<typename Policy<M>::R, PT> A) {
  using R = typename Policy<M>::R;
  using RayT = Ray<M, PT, NF>;
  using Item = ItemDesc<R, PT>;
  constexpr unsigned kFull = 0xffffffffu;
  const unsigned lane = threadIdx.x & 31u;
  RayT ray;
  RayCounters ctr{};
  const Item* d = nullptr;
  bool live = false;
  unsigned long long claim = kNoClaim;
  unsigned long long steps = 0, nplasma = 0, bad = 0, rays = 0;
  long long idle = 0;
  const unsigned long long tile_rays = (unsigned long long)A.tile_rays;
  for (;;) {
    // claim slots for lanes that have neither a ray nor a claim; start every claim whose tile is published
    const unsigned need = __ballot_sync(kFull, !live && claim == kNoClaim);
    if (need) {
      unsigned long long base = 0;
      if (lane == 0) base = atomicAdd(&A.ctl[kQHead], (unsigned long long)__popc(need));
      base = __shfl_sync(kFull, base, 0);
      if (!live && claim == kNoClaim) claim = base + __popc(need & ((1u << lane) - 1u));
    }
    unsigned long long tail = 0;
    if (lane == 0) tail = ld_acquire_u64(&A.ctl[kQTail]);
    tail = __shfl_sync(kFull, tail, 0) * tile_rays;
    if (!live && claim != kNoClaim && claim < tail) {
      const unsigned long long t = claim / tile_rays;
      const int off = (int)(claim - t * tile_rays);
      const int4 raw = __ldcg(reinterpret_cast<const int4*>(A.tiles + (t & A.tile_mask)));
      claim = kNoClaim;
      if (off < raw.z) {
        d = A.items + raw.x;
        const int32_t pix = d->jobs[raw.y + off];
        if (pix >= 0 && pix < d->rc.W * d->rc.H) {
          if (d->starts) {
            ray.init_from(d->starts[raw.y + off], pix);
          } else {
            ray.init(d->snap, d->snap_d, d->rc, pix);
          }
          live = true;
        }
      }
    }
    if (!__any_sync(kFull, live)) {
      // every lane idle: claims past the tail (drained or not yet published), or a slot that held no job
      const bool beyond = claim != kNoClaim;
      if (A.idle_ns == 0) {
        if (__all_sync(kFull, beyond)) break;
        continue;
      }
      unsigned long long stop = 0;
      if (lane == 0) stop = ld_volatile_u64(&A.ctl[kQStop]);
      if (__shfl_sync(kFull, stop, 0)) break;
      if (++idle > A.idle_limit) {
        if (lane == 0) atomicMax(&A.ctl[kQStatus], 1ull);
        break;
      }
      if (__all_sync(kFull, beyond)) __nanosleep((unsigned)A.idle_ns);
      continue;
    }
    idle = 0;
    for (int it = 0; it < A.period; it++) {
      if (live) {
        live = ray.advance(d->snap, d->snap_d, d->rc, ctr);
        if (!live) {
          ray.write(d->out, d->rc.nfreqs);
          if (d->pixstats) {
            int32_t* ps = d->pixstats + 3 * (size_t)ray.pix;
            ps[0] = ray.steps;
            ps[1] = ray.nplasma;
            ps[2] = ray.bad;
          }
          steps += (unsigned)ray.steps;
          nplasma += (unsigned)ray.nplasma;
          bad += (unsigned)ray.bad;
          rays++;
          atomicAdd(&d->ctr[kItSteps], (unsigned long long)ray.steps);
          atomicAdd(&d->ctr[kItPlasma], (unsigned long long)ray.nplasma);
          if (ray.bad) atomicAdd(&d->ctr[kItBad], (unsigned long long)ray.bad);
          __threadfence();
          const unsigned long long n = atomicAdd(&d->ctr[kItRays], 1ull);
          if (n + 1 == d->nrays && d->done) {
            __threadfence_system();
            *d->done = 1;
          }
        }
      }
      // a warp with refill_lanes finished lanes claims new slots at once instead of at the end of the period
      if ((it & 63) == 63 && __popc(__ballot_sync(kFull, !live)) >= A.refill_lanes) break;
    }
  }
  steps = warp_sum_u64(steps);
  nplasma = warp_sum_u64(nplasma);
  bad = warp_sum_u64(bad);
  rays = warp_sum_u64(rays);
  const unsigned long long scans = warp_sum_u64(ctr.scans);
  const unsigned long long f64s = warp_sum_u64(ctr.fp64_steps);
  const unsigned long long f64o = warp_sum_u64(ctr.fp64_ops);
  if (lane == 0) {
    atomicAdd(&A.counters[kCtrSteps], steps);
    atomicAdd(&A.counters[kCtrPlasma], nplasma);
    atomicAdd(&A.counters[kCtrBad], bad);
    atomicAdd(&A.counters[kCtrRays], rays);
    if (scans) atomicAdd(&A.counters[kCtrScans], scans);
    if (f64s) atomicAdd(&A.counters[kCtrFp64Steps], f64s);
    if (f64o) atomicAdd(&A.counters[kCtrFp64Ops], f64o);
  }
}

// The camera set-up of every job of one image (the batched tile generator's ray set-up): one thread per job, all lanes
// busy, written in job order for the queue kernel's refills to read.  G: the geodesic precision of the mode, whose
// ray_start the march would call (the same out-of-line function, so rays start bit-identically).
template <class G, class R>
__global__ void __launch_bounds__(128) k_ray_setup(const __grid_constant__ RenderConsts<R> rc, G a, G hs,
                                                   const int32_t* __restrict__ jobs, long long njobs,
                                                   RayStart* __restrict__ out) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < njobs; k += stride) {
    const int32_t pix = jobs[k];
    if (pix >= 0 && pix < rc.W * rc.H) out[k] = ray_start<G>(rc, a, hs, pix);
  }
}

// Launches k_ray_setup for one image of mode M (instantiated beside that mode's queue kernels, with their flags).
template <Mode M, class PT>
cudaError_t launch_ray_setup(const ItemDesc<typename Policy<M>::R, PT>& item, long long njobs, int sms,
                             RayStart* out, cudaStream_t stream);

// Launch configuration of the queue kernel (the autotuner's search space).
struct QueueShape {
  int blocks_per_sm;  // register-cap variant: 1, 3 or 4 (FP32); mixed 1, 3 (4 with one slot); FP64 1; 0 = default
  int period;
  int refill_lanes;   // 1..32 (0: 32, when the warp is empty)
};

// Default register-cap variant (measured on B200): FP32 128 registers (16 warps per SM); mixed 128 with one frequency
// slot (330 ms vs 368 ms at 168 registers on the 128-image sweep's autotuning sample), else 168 (12 warps); FP64
// uncapped.
template <Mode M, int NF>
constexpr int default_queue_blocks_per_sm() {
  return M == Mode::kFP32 ? 4 : M == Mode::kMixed ? (NF == 1 ? 4 : 3) : 1;
}

// Launches the queue kernel for `nf_slots` frequency slots (1, 4 or 32) on a persistent grid (resident blocks x SMs),
// capped at the blocks `max_rays` rays can fill when max_rays > 0.
template <Mode M, class PT>
cudaError_t launch_queue(const QueueArgs<typename Policy<M>::R, PT>& args, int nf_slots, int sms, QueueShape q,
                         long long max_rays, cudaStream_t stream, LaunchShape* shape);

// Resets a queue's control words (head 0, tail = ntiles, stop and status 0), a kernel-wide counter block and
// n_item_words item counters, on the stream: the first node of a captured batch.
cudaError_t launch_queue_reset(unsigned long long* ctl, unsigned long long* counters, unsigned long long* item_ctr,
                               long long n_item_words, unsigned long long ntiles, cudaStream_t stream);

}  // namespace phx
