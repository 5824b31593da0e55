// Batches: many images rendered by one persistent launch of the queue kernel (queue.cuh), captured in a CUDA graph.
//
// Creation uploads every item's constants (camera, integration, plasma, frequencies), its snapshot view and its job
// list, allocates the results, cuts the job lists into tiles of `tile_rays` rays (the largest images first unless the
// caller keeps its order: their long rays start early and short images fill the end), optionally autotunes the launch
// (register-cap variant x refill period, each timed on an every-n-th-tile sample of the batch, then the tile shapes)
// and captures [queue reset, ray set-up of every item, queue kernel] into a graph that phx_batch_launch replays.  The
// ray set-up (k_ray_setup, the camera photon and polarization of every job at full SIMD width) replaces the set-up a
// lane would otherwise run alone, with most of its warp idle, each time it takes a new ray.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <functional>
#include <numeric>
#include <string>
#include <vector>

#include "internal.hpp"
#include "queue.cuh"

using namespace phx_capi;

struct PhxBatch {
  int device = 0, sms = 0;
  int32_t precision = PHX_PREC_FP32;
  int nf_slots = 1;
  std::vector<PhxRenderParams> params;
  std::vector<int64_t> njobs;
  std::vector<size_t> out_off;  // record offsets into out
  std::vector<size_t> job_off;  // job-list offsets into jobs
  std::vector<char> own_order;  // item's job list is the batch's pixel order (no caller job list)
  int tile_shape = PHX_TILE_MORTON;
  void* items = nullptr;
  phx::TileDesc* tiles = nullptr;
  phx::TileDesc* trial = nullptr;
  int64_t ntiles = 0, ntrial = 0, nrays = 0, trial_rays = 0;
  unsigned tile_mask = 0, trial_mask = 0;
  int32_t* jobs = nullptr;
  PhxFreqOut* out = nullptr;
  PhxSpectrum* spec = nullptr;  // per-frequency totals of one item (phx_batch_spectrum)
  phx::RayStart* starts = nullptr;  // camera set-up of every job (job order), or null: lanes set up their rays
  size_t nrecords = 0;
  unsigned long long* item_ctr = nullptr;
  unsigned long long* ctl = nullptr;
  unsigned long long* counters = nullptr;
  int tile_rays = 32;
  phx::QueueShape shape{3, 32};
  phx::LaunchShape lshape{};
  PhxBatchTuning tuning{};
  int64_t device_bytes = 0;
  double kernel_s = 0.0;
  // launches the queue kernel over (tiles, ntiles published, mask) with a shape, on a stream
  std::function<cudaError_t(const phx::TileDesc*, unsigned, phx::QueueShape, long long, cudaStream_t,
                            phx::LaunchShape*)>
      launch;
  // launches the ray-setup kernel of every item on a stream (empty without a start-state buffer)
  std::function<cudaError_t(cudaStream_t)> setup;
  cudaStream_t stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  std::vector<void*> owned;

  template <class T>
  T* alloc(size_t n) {
    T* p = nullptr;
    ck(cudaMalloc((void**)&p, std::max<size_t>(n, 1) * sizeof(T)), "cudaMalloc");
    owned.push_back(p);
    device_bytes += (int64_t)(std::max<size_t>(n, 1) * sizeof(T));
    return p;
  }

  ~PhxBatch() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (stream) cudaStreamDestroy(stream);
    for (void* p : owned) cudaFree(p);
  }
};

namespace {

// Pixel order of a W x H image for a tile shape (PHX_TILE_*, phx_schedule_tiles).
std::vector<int32_t> pixel_order(int32_t W, int32_t H, int shape) {
  std::vector<int32_t> m((size_t)W * H);
  if (phx_schedule_tiles(W, H, shape, m.data()) != PHX_OK) throw std::runtime_error(last_error());
  return m;
}

// Writes every own-order item's job list for `shape` into the device job array.
void upload_order(PhxBatch* b, int shape) {
  for (size_t i = 0; i < b->params.size(); i++) {
    if (!b->own_order[i]) continue;
    const std::vector<int32_t> m = pixel_order(b->params[i].img_width, b->params[i].img_height, shape);
    ck(cudaMemcpy(b->jobs + b->job_off[i], m.data(), m.size() * sizeof(int32_t), cudaMemcpyHostToDevice), "H2D jobs");
  }
  b->tile_shape = shape;
}

unsigned pow2_mask(int64_t n) {
  unsigned long long c = 1;
  while ((long long)c < n) c <<= 1;
  if (c > (1ull << 31)) throw std::invalid_argument("batch too large (more than 2^31 tiles)");
  return (unsigned)(c - 1);
}

// Item table of mode M and the launcher bound to it.
template <phx::Mode M, class PT>
void build_items(PhxBatch* b, const PhxBatchItem* items, int32_t nitems, const std::vector<size_t>& job_off) {
  using R = typename phx::Policy<M>::R;
  using Item = phx::ItemDesc<R, PT>;
  std::vector<Item> h(nitems);
  for (int32_t i = 0; i < nitems; i++) {
    std::memset((void*)&h[i], 0, sizeof(Item));
    const PhxSnapshot* s = items[i].snapshot;
    h[i].rc = phx::make_consts<R>(b->params[i], s->a, s->hslope);
    h[i].snap = view_for<M, PT>(s);
    h[i].snap_d = h[i].snap.fp64_view();
    h[i].jobs = b->jobs + job_off[i];
    h[i].starts = b->starts ? b->starts + job_off[i] : nullptr;
    h[i].out = reinterpret_cast<double*>(b->out + b->out_off[i]);
    h[i].pixstats = nullptr;
    h[i].ctr = b->item_ctr + (size_t)phx::kItemCounters * i;
    h[i].nrays = (unsigned long long)b->njobs[i];
    h[i].done = nullptr;
  }
  Item* d = b->alloc<Item>(nitems);
  ck(cudaMemcpy(d, h.data(), sizeof(Item) * nitems, cudaMemcpyHostToDevice), "H2D items");
  b->items = d;
  const int nf = b->nf_slots, sms = b->sms;
  unsigned long long* ctl = b->ctl;
  unsigned long long* counters = b->counters;
  const int tile_rays = b->tile_rays;
  if (b->starts) {
    std::vector<int64_t> njobs = b->njobs;
    b->setup = [h, njobs, sms](cudaStream_t st) -> cudaError_t {
      for (size_t i = 0; i < h.size(); i++) {
        const cudaError_t e = phx::launch_ray_setup<M, PT>(h[i], njobs[i], sms, const_cast<phx::RayStart*>(h[i].starts),
                                                            st);
        if (e != cudaSuccess) return e;
      }
      return cudaSuccess;
    };
  }
  b->launch = [d, nf, sms, ctl, counters, tile_rays](const phx::TileDesc* tiles, unsigned mask, phx::QueueShape q,
                                                      long long max_rays, cudaStream_t st, phx::LaunchShape* ls) {
    phx::QueueArgs<R, PT> A;
    A.items = d;
    A.tiles = tiles;
    A.ctl = ctl;
    A.counters = counters;
    A.tile_mask = mask;
    A.tile_rays = tile_rays;
    A.period = q.period;
    A.idle_ns = 0;
    A.idle_limit = 0;
    return phx::launch_queue<M, PT>(A, nf, sms, q, max_rays, st, ls);
  };
}

// One timed launch over `ntiles` tiles of `tiles` (reset + kernel) on the batch stream; returns milliseconds.
float timed_launch(PhxBatch* b, const phx::TileDesc* tiles, int64_t ntiles, unsigned mask, long long max_rays,
                   phx::QueueShape q, phx::LaunchShape* ls) {
  const long long nwords = (long long)phx::kItemCounters * (long long)b->params.size();
  ck(phx::launch_queue_reset(b->ctl, b->counters, b->item_ctr, nwords, (unsigned long long)ntiles, b->stream),
     "queue reset");
  ck(cudaEventRecord(b->e0, b->stream), "event");
  ck(b->launch(tiles, mask, q, max_rays, b->stream, ls), "queue launch");
  ck(cudaEventRecord(b->e1, b->stream), "event");
  ck(cudaStreamSynchronize(b->stream), "batch trial");
  float ms = 0.f;
  ck(cudaEventElapsedTime(&ms, b->e0, b->e1), "event time");
  return ms;
}

// Sets up every job's camera ray now (autotuning trials time the queue kernel alone).
void run_setup(PhxBatch* b) {
  if (!b->setup) return;
  ck(b->setup(b->stream), "ray setup");
  ck(cudaStreamSynchronize(b->stream), "ray setup");
}

void autotune(PhxBatch* b) {
  std::vector<phx::QueueShape> cand;
  // refill policies: the finished lanes every 128 passes; a warp with 24 finished lanes; a warp with all 32 finished
  const int policies[3][2] = {{128, 1}, {phx::kDefaultQueuePeriod, 24}, {phx::kDefaultQueuePeriod, 32}};
  auto add = [&](int bps) {
    for (const auto& pol : policies) cand.push_back({bps, pol[0], pol[1]});
  };
  if (b->precision == PHX_PREC_FP32 && b->nf_slots <= 4) {
    for (int bps : {3, 4, 1}) add(bps);
  } else if (b->precision == PHX_PREC_MIXED && b->nf_slots == 1) {
    for (int bps : {3, 4, 1}) add(bps);
  } else if (b->precision == PHX_PREC_MIXED) {
    for (int bps : {3, 1}) add(bps);
  } else {
    add(0);
  }
  // load every variant once (an empty queue: the kernel leaves at its first refill)
  phx::LaunchShape ls;
  for (const auto& q : cand) timed_launch(b, b->trial, 0, b->trial_mask, 1, q, &ls);
  int nc = 0;
  auto record = [&](const phx::QueueShape& q, int shape, float ms) {
    if (nc >= PHX_TUNE_MAX_CANDIDATES) return;
    b->tuning.cand_blocks_per_sm[nc] = q.blocks_per_sm;
    b->tuning.cand_period[nc] = q.period;
    b->tuning.cand_refill_lanes[nc] = q.refill_lanes;
    b->tuning.cand_tile_shape[nc] = shape;
    b->tuning.cand_ms[nc] = ms;
    nc++;
  };
  // stage 1: register cap x refill policy, in the current pixel order
  const int shape0 = b->tile_shape;
  float best = 1e30f;
  for (size_t c = 0; c < cand.size(); c++) {
    const float ms = timed_launch(b, b->trial, b->ntrial, b->trial_mask, b->trial_rays, cand[c], &ls);
    record(cand[c], shape0, ms);
    if (ms < best) {
      best = ms;
      b->shape = cand[c];
    }
  }
  // stage 2: the other tile shapes at the best launch shape (only items without a caller job list change order)
  const bool any_own = std::any_of(b->own_order.begin(), b->own_order.end(), [](char c) { return c != 0; });
  int best_shape = shape0;
  if (any_own) {
    for (int shape = 0; shape < PHX_TILE_SHAPES; shape++) {
      if (shape == shape0) continue;
      upload_order(b, shape);
      run_setup(b);
      const float ms = timed_launch(b, b->trial, b->ntrial, b->trial_mask, b->trial_rays, b->shape, &ls);
      record(b->shape, shape, ms);
      if (ms < best) {
        best = ms;
        best_shape = shape;
      }
    }
    if (b->tile_shape != best_shape) upload_order(b, best_shape);
  }
  b->tuning.ncand = nc;
}

void capture(PhxBatch* b) {
  const long long nwords = (long long)phx::kItemCounters * (long long)b->params.size();
  ck(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeRelaxed), "begin capture");
  cudaError_t e = phx::launch_queue_reset(b->ctl, b->counters, b->item_ctr, nwords, (unsigned long long)b->ntiles,
                                          b->stream);
  if (e == cudaSuccess && b->setup) e = b->setup(b->stream);
  if (e == cudaSuccess) e = b->launch(b->tiles, b->tile_mask, b->shape, b->nrays, b->stream, &b->lshape);
  cudaGraph_t g = nullptr;
  const cudaError_t e2 = cudaStreamEndCapture(b->stream, &g);
  ck(e, "captured batch launch");
  ck(e2, "end capture");
  b->graph = g;
  ck(cudaGraphInstantiate(&b->exec, b->graph, 0), "graph instantiate");
}

PhxBatch* create_batch(const PhxBatchItem* items, int32_t nitems, const PhxBatchOptions* opt) {
  if (!items || nitems < 1) throw std::invalid_argument("a batch needs at least one item");
  PhxBatchOptions o;
  phx_default_batch_options(&o);
  if (opt) o = *opt;
  if (o.tile_rays <= 0) o.tile_rays = 32;
  if (o.tile_rays > 4096) throw std::invalid_argument("tile_rays must be <= 4096");
  if (o.sample_stride <= 0) o.sample_stride = 16;
  auto b = std::make_unique<PhxBatch>();
  ck(cudaGetDevice(&b->device), "cudaGetDevice");
  b->tile_rays = o.tile_rays;
  b->precision = items[0].params.precision;
  int maxf = 1;
  bool f64prims = true;
  for (int32_t i = 0; i < nitems; i++) {
    const PhxBatchItem& it = items[i];
    if (!it.snapshot) throw std::invalid_argument("item " + std::to_string(i) + ": null snapshot");
    if (it.snapshot->device != b->device) throw std::invalid_argument("every item's snapshot must live on the current device");
    phx::check_params(it.params);
    if (it.params.precision != b->precision) throw std::invalid_argument("every item of a batch needs the same precision");
    maxf = std::max(maxf, (int)it.params.nfreqs);
    f64prims = f64prims && it.snapshot->prim_d;
    b->sms = it.snapshot->sms;
  }
  b->nf_slots = maxf <= 1 ? 1 : maxf <= 4 ? 4 : phx::kMaxFreqs;
  if (b->nf_slots > 4 && b->precision != PHX_PREC_FP32)
    throw std::invalid_argument("batches with more than 4 frequencies per image are FP32 only");
  // job lists (validated) and result offsets
  if (o.tile_shape < 0 || o.tile_shape >= PHX_TILE_SHAPES) throw std::invalid_argument("unknown tile_shape");
  if (o.refill_lanes < 0 || o.refill_lanes > 32) throw std::invalid_argument("refill_lanes must be in 0..32");
  b->tile_shape = o.tile_shape;
  std::vector<int32_t> all_jobs;
  std::vector<size_t>& job_off = b->job_off;
  job_off.assign(nitems, 0);
  b->own_order.assign(nitems, 0);
  b->params.resize(nitems);
  b->njobs.resize(nitems);
  b->out_off.resize(nitems);
  size_t nrec = 0;
  for (int32_t i = 0; i < nitems; i++) {
    const PhxRenderParams& p = items[i].params;
    b->params[i] = p;
    const int64_t npix = (int64_t)p.img_width * p.img_height;
    job_off[i] = all_jobs.size();
    if (items[i].jobs) {
      if (items[i].njobs < 0 || items[i].njobs > npix) throw std::invalid_argument("njobs out of range");
      for (int64_t n = 0; n < items[i].njobs; n++) {
        const int32_t j = items[i].jobs[n];
        if (j < 0 || j >= npix) throw std::invalid_argument("job index out of range");
        all_jobs.push_back(j);
      }
      b->njobs[i] = items[i].njobs;
    } else {
      const std::vector<int32_t> m = pixel_order(p.img_width, p.img_height, b->tile_shape);
      all_jobs.insert(all_jobs.end(), m.begin(), m.end());
      b->njobs[i] = npix;
      b->own_order[i] = 1;
    }
    nrec = (nrec + 3) & ~(size_t)3;  // 192-byte aligned records per item
    b->out_off[i] = nrec;
    nrec += (size_t)npix * p.nfreqs;
  }
  b->nrecords = nrec;
  // tiles: the largest images first unless the caller keeps its order
  std::vector<int32_t> order(nitems);
  std::iota(order.begin(), order.end(), 0);
  if (!o.keep_order)
    std::stable_sort(order.begin(), order.end(), [&](int32_t x, int32_t y) { return b->njobs[x] > b->njobs[y]; });
  std::vector<phx::TileDesc> tiles;
  for (int32_t i : order)
    for (int64_t f = 0; f < b->njobs[i]; f += o.tile_rays)
      tiles.push_back({i, (int32_t)f, (int32_t)std::min<int64_t>(o.tile_rays, b->njobs[i] - f), 0});
  b->ntiles = (int64_t)tiles.size();
  b->nrays = std::accumulate(b->njobs.begin(), b->njobs.end(), (int64_t)0);
  std::vector<phx::TileDesc> trial;
  for (size_t t = 0; t < tiles.size(); t += o.sample_stride) {
    trial.push_back(tiles[t]);
    b->trial_rays += tiles[t].count;
  }
  b->ntrial = (int64_t)trial.size();
  b->tile_mask = pow2_mask(std::max<int64_t>(b->ntiles, 1));
  b->trial_mask = pow2_mask(std::max<int64_t>(b->ntrial, 1));
  // device buffers
  b->jobs = b->alloc<int32_t>(all_jobs.size());
  if (!all_jobs.empty())
    ck(cudaMemcpy(b->jobs, all_jobs.data(), all_jobs.size() * sizeof(int32_t), cudaMemcpyHostToDevice), "H2D jobs");
  b->out = b->alloc<PhxFreqOut>(nrec);
  if (!o.lane_setup) b->starts = b->alloc<phx::RayStart>(all_jobs.size());
  ck(cudaMemset(b->out, 0, std::max<size_t>(nrec, 1) * sizeof(PhxFreqOut)), "memset results");
  b->item_ctr = b->alloc<unsigned long long>((size_t)phx::kItemCounters * nitems);
  b->ctl = b->alloc<unsigned long long>(phx::kQWords);
  b->counters = b->alloc<unsigned long long>(phx::kNumCounters);
  b->tiles = b->alloc<phx::TileDesc>((size_t)b->tile_mask + 1);
  if (!tiles.empty())
    ck(cudaMemcpy(b->tiles, tiles.data(), tiles.size() * sizeof(phx::TileDesc), cudaMemcpyHostToDevice), "H2D tiles");
  b->trial = b->alloc<phx::TileDesc>((size_t)b->trial_mask + 1);
  if (!trial.empty())
    ck(cudaMemcpy(b->trial, trial.data(), trial.size() * sizeof(phx::TileDesc), cudaMemcpyHostToDevice), "H2D tiles");
  switch (b->precision) {
    case PHX_PREC_FP32:
      build_items<phx::Mode::kFP32, float>(b.get(), items, nitems, job_off);
      break;
    case PHX_PREC_MIXED:
      build_items<phx::Mode::kMixed, float>(b.get(), items, nitems, job_off);
      break;
    case PHX_PREC_FP64:
      if (f64prims) build_items<phx::Mode::kFP64, double>(b.get(), items, nitems, job_off);
      else build_items<phx::Mode::kFP64, float>(b.get(), items, nitems, job_off);
      break;
    default:
      throw std::invalid_argument("unknown precision");
  }
  ck(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "cudaStreamCreate");
  ck(cudaEventCreate(&b->e0), "cudaEventCreate");
  ck(cudaEventCreate(&b->e1), "cudaEventCreate");
  b->shape = {o.blocks_per_sm > 0
                  ? o.blocks_per_sm
                  : (b->precision == PHX_PREC_FP32 ? 4 : b->precision == PHX_PREC_MIXED ? (b->nf_slots == 1 ? 4 : 3) : 1),
              o.period > 0 ? o.period : phx::kDefaultQueuePeriod, o.refill_lanes > 0 ? o.refill_lanes : 32};
  run_setup(b.get());
  if (o.autotune && b->ntrial > 0) autotune(b.get());
  capture(b.get());
  b->tuning.blocks_per_sm = b->shape.blocks_per_sm;
  b->tuning.period = b->shape.period;
  b->tuning.refill_lanes = b->shape.refill_lanes;
  b->tuning.tile_rays = b->tile_rays;
  b->tuning.tile_shape = b->tile_shape;
  b->tuning.grid = b->lshape.grid;
  b->tuning.block = b->lshape.block;
  b->tuning.regs = b->lshape.regs;
  b->tuning.local_bytes = b->lshape.local_bytes;
  b->tuning.nitems = nitems;
  b->tuning.ntiles = b->ntiles;
  b->tuning.nrays = b->nrays;
  b->tuning.device_bytes = b->device_bytes;
  return b.release();
}

}  // namespace

extern "C" {

void phx_default_batch_options(PhxBatchOptions* o) {
  if (!o) return;
  std::memset(o, 0, sizeof *o);
  o->tile_rays = 32;
  o->sample_stride = 16;
}

int phx_batch_create(const PhxBatchItem* items, int32_t nitems, const PhxBatchOptions* opt, PhxBatch** out) {
  return guarded([&]() -> int {
    if (!out) throw std::invalid_argument("null output handle");
    *out = create_batch(items, nitems, opt);
    return PHX_OK;
  });
}

int phx_batch_launch(PhxBatch* b, void* stream) {
  return guarded([&]() -> int {
    if (!b) throw std::invalid_argument("null batch");
    ck(cudaGraphLaunch(b->exec, (cudaStream_t)stream), "batch graph launch");
    return PHX_OK;
  });
}

int phx_batch_run(PhxBatch* b) {
  return guarded([&]() -> int {
    if (!b) throw std::invalid_argument("null batch");
    ck(cudaEventRecord(b->e0, b->stream), "event");
    ck(cudaGraphLaunch(b->exec, b->stream), "batch graph launch");
    ck(cudaEventRecord(b->e1, b->stream), "event");
    ck(cudaStreamSynchronize(b->stream), "batch run");
    float ms = 0.f;
    ck(cudaEventElapsedTime(&ms, b->e0, b->e1), "event time");
    b->kernel_s = ms * 1e-3;
    return PHX_OK;
  });
}

int phx_batch_result(PhxBatch* b, int32_t item, PhxFreqOut* res, PhxRenderInfo* info) {
  return guarded([&]() -> int {
    if (!b || !res) throw std::invalid_argument("null argument");
    if (item < 0 || item >= (int32_t)b->params.size()) throw std::invalid_argument("item out of range");
    const PhxRenderParams& p = b->params[item];
    const size_t n = (size_t)p.img_width * p.img_height * p.nfreqs;
    ck(cudaMemcpy(res, b->out + b->out_off[item], n * sizeof(PhxFreqOut), cudaMemcpyDeviceToHost), "D2H results");
    if (info) {
      unsigned long long c[phx::kItemCounters];
      ck(cudaMemcpy(c, b->item_ctr + (size_t)phx::kItemCounters * item, sizeof c, cudaMemcpyDeviceToHost),
         "D2H counters");
      std::memset(info, 0, sizeof *info);
      cudaDeviceProp prop;
      ck(cudaGetDeviceProperties(&prop, b->device), "cudaGetDeviceProperties");
      std::snprintf(info->device, sizeof info->device, "%.200s (sm_%d%d)", prop.name, prop.major, prop.minor);
      info->sms = b->sms;
      info->blocks = b->lshape.grid;
      info->block = b->lshape.block;
      info->regs = b->lshape.regs;
      info->local_bytes = b->lshape.local_bytes;
      info->kernel_s = b->kernel_s;
      info->steps = (int64_t)c[phx::kItSteps];
      info->nplasma = (int64_t)c[phx::kItPlasma];
      info->bad = (int64_t)c[phx::kItBad];
    }
    return PHX_OK;
  });
}

int phx_batch_device_result(PhxBatch* b, int32_t item, PhxFreqOut** d_res) {
  return guarded([&]() -> int {
    if (!b || !d_res) throw std::invalid_argument("null argument");
    if (item < 0 || item >= (int32_t)b->params.size()) throw std::invalid_argument("item out of range");
    *d_res = b->out + b->out_off[item];
    return PHX_OK;
  });
}

int phx_batch_spectrum(PhxBatch* b, int32_t item, PhxSpectrum* spec) {
  return guarded([&]() -> int {
    if (!b || !spec) throw std::invalid_argument("null argument");
    if (item < 0 || item >= (int32_t)b->params.size()) throw std::invalid_argument("item out of range");
    const PhxRenderParams& p = b->params[item];
    if (!b->spec) b->spec = b->alloc<PhxSpectrum>(PHX_MAX_FREQS);
    launch_spectrum(p, b->out + b->out_off[item], b->spec, b->stream);
    ck(cudaMemcpyAsync(spec, b->spec, p.nfreqs * sizeof(PhxSpectrum), cudaMemcpyDeviceToHost, b->stream),
       "D2H spectrum");
    ck(cudaStreamSynchronize(b->stream), "spectrum");
    return PHX_OK;
  });
}

int phx_batch_tuning(const PhxBatch* b, PhxBatchTuning* t) {
  return guarded([&]() -> int {
    if (!b || !t) throw std::invalid_argument("null argument");
    *t = b->tuning;
    return PHX_OK;
  });
}

void phx_batch_destroy(PhxBatch* b) { delete b; }

}  // extern "C"
