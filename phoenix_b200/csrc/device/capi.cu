// The extern "C" boundary (include/phoenix_b200.h): snapshot residency, render launches, errors.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <cmath>
#include <exception>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../../include/phoenix_b200.h"
#include "../host/output.hpp"
#include "../host/render_setup.hpp"
#include "../host/snapshot.hpp"
#include "internal.hpp"
#include "march.cuh"

using namespace phx_capi;

namespace {

template <phx::Mode M, class PT>
cudaError_t launch_mode(PhxSnapshot* s, const PhxRenderParams& p, const typename phx::Policy<M>::R* lb,
                        const typename phx::Policy<M>::R* dxc, const PT* prim, const int32_t* d_jobs, int64_t njobs,
                        PhxFreqOut* d_res, int32_t* d_pixstats, uint64_t* d_counters, cudaStream_t st,
                        phx::LaunchShape* shape) {
  using R = typename phx::Policy<M>::R;
  phx::MarchArgs<R, PT> A;
  A.snap = snap_view<R, PT>(s, lb, dxc, prim);
  A.snap_d = A.snap.fp64_view();
  A.rc = phx::make_consts<R>(p, s->a, s->hslope);
  A.jobs = d_jobs;
  A.njobs = njobs;
  A.out = reinterpret_cast<double*>(d_res);
  A.pixstats = d_pixstats;
  A.counters = reinterpret_cast<unsigned long long*>(d_counters);
  A.period = p.period > 0 ? p.period : phx::kDefaultPeriod;  // passes between lane refills (measured best on B200)
  A.refill_lanes = p.refill_lanes > 0 ? p.refill_lanes : 32;
  return phx::launch_march<M, PT>(A, s->sms, p.blocks_per_sm, st, shape);
}

cudaError_t dispatch(PhxSnapshot* s, const PhxRenderParams& p, const int32_t* d_jobs, int64_t njobs, PhxFreqOut* d_res,
                     int32_t* d_pixstats, uint64_t* d_counters, cudaStream_t st, phx::LaunchShape* shape) {
  switch (p.precision) {
    case PHX_PREC_FP32:
      return launch_mode<phx::Mode::kFP32, float>(s, p, s->lb_f, s->dxc_f, s->prim_f, d_jobs, njobs, d_res, d_pixstats,
                                                  d_counters, st, shape);
    case PHX_PREC_MIXED:
      return launch_mode<phx::Mode::kMixed, float>(s, p, s->lb_f, s->dxc_f, s->prim_f, d_jobs, njobs, d_res,
                                                   d_pixstats, d_counters, st, shape);
    case PHX_PREC_FP64:
      if (s->prim_d)
        return launch_mode<phx::Mode::kFP64, double>(s, p, s->lb_d, s->dxc_d, s->prim_d, d_jobs, njobs, d_res,
                                                     d_pixstats, d_counters, st, shape);
      return launch_mode<phx::Mode::kFP64, float>(s, p, s->lb_d, s->dxc_d, s->prim_f, d_jobs, njobs, d_res,
                                                  d_pixstats, d_counters, st, shape);
  }
  return cudaErrorInvalidValue;
}

void validate_desc(const PhxSnapshotDesc* d, bool defer_prims = false) {
  auto bad = [](const std::string& m) { throw std::invalid_argument(m); };
  if (!d) bad("null snapshot descriptor");
  if (d->nleafs < 1) bad("nleafs must be >= 1");
  if (d->nlevels < 1 || d->nlevels > PHX_MAX_LEVELS) bad("nlevels must be in 1..16");
  for (int k = 0; k < 3; k++) {
    if (d->nx[k] < 1 || d->ng[k] < 1) bad("nx and ng must be positive");
    if (!(d->x_hi[k] > d->x_lo[k])) bad("empty domain");
  }
  if (!d->lb || !d->dxc || (!d->prim_f32 && !defer_prims) || !d->level_map)
    bad("lb, dxc, prim_f32 and level_map are required");
  if (!(std::fabs(d->a) < 1.0)) bad("spin must satisfy |a| < 1");
  const size_t top = (size_t)1 << (d->nlevels - 1);
  const size_t slots = d->ng[0] * top * d->ng[1] * top * d->ng[2] * top;
  if (slots > ((size_t)1 << 31)) bad("finest-level leaf map too large (> 2^31 slots)");
  for (int L = 0; L < d->nlevels; L++) {
    if (!d->level_map[L]) bad("level_map[" + std::to_string(L) + "] is null");
    const size_t n = ((size_t)d->ng[0] << L) * ((size_t)d->ng[1] << L) * ((size_t)d->ng[2] << L);
    for (size_t t = 0; t < n; t++) {
      const int32_t v = d->level_map[L][t];
      if (v < -1 || v >= d->nleafs) bad("level_map holds a leaf id out of range");
    }
  }
}

// defer_prims: allocate the primitive pool without filling it (the GPU decode writes it).
PhxSnapshot* create_snapshot(const PhxSnapshotDesc* d, int32_t flags, bool defer_prims = false) {
  validate_desc(d, defer_prims);
  const auto t0 = std::chrono::steady_clock::now();
  auto s = std::make_unique<PhxSnapshot>();
  ck(cudaGetDevice(&s->device), "cudaGetDevice");
  cudaDeviceProp prop;
  ck(cudaGetDeviceProperties(&prop, s->device), "cudaGetDeviceProperties");
  s->sms = prop.multiProcessorCount;
  std::snprintf(s->device_name, sizeof s->device_name, "%s (sm_%d%d)", prop.name, prop.major, prop.minor);
  s->nleafs = d->nleafs;
  s->nlevels = d->nlevels;
  s->cells = d->nx[0] * d->nx[1] * d->nx[2];
  s->a = d->a;
  s->hslope = d->hslope;
  s->gam = d->gam;
  for (int k = 0; k < 3; k++) {
    s->nx[k] = d->nx[k];
    s->ng[k] = d->ng[k];
    s->fd[k] = d->ng[k] << (d->nlevels - 1);
    s->x_lo[k] = d->x_lo[k];
    s->x_hi[k] = d->x_hi[k];
  }
  const size_t n3 = 3 * (size_t)d->nleafs;
  std::vector<float> lbf(n3), dxf(n3);
  for (size_t t = 0; t < n3; t++) {
    lbf[t] = (float)d->lb[t];
    dxf[t] = (float)d->dxc[t];
  }
  std::vector<std::vector<int32_t>> maps(d->nlevels);
  for (int L = 0; L < d->nlevels; L++) {
    const size_t n = ((size_t)d->ng[0] << L) * ((size_t)d->ng[1] << L) * ((size_t)d->ng[2] << L);
    maps[L].assign(d->level_map[L], d->level_map[L] + n);
  }
  const std::vector<int32_t> flat = phx::flatten_level_maps(maps, d->ng, d->nlevels);
  const size_t nprim = (size_t)d->nleafs * s->cells * phx::kNPrim;
  s->lb_f = dev_upload(lbf.data(), n3, s->owned);
  s->dxc_f = dev_upload(dxf.data(), n3, s->owned);
  s->lb_d = dev_upload(d->lb, n3, s->owned);
  s->dxc_d = dev_upload(d->dxc, n3, s->owned);
  if (defer_prims) {
    ck(cudaMalloc((void**)&s->prim_f, nprim * sizeof(float)), "cudaMalloc primitives");
    s->owned.push_back(s->prim_f);
    if (flags & PHX_SNAP_F64_PRIMS) {
      ck(cudaMalloc((void**)&s->prim_d, nprim * sizeof(double)), "cudaMalloc primitives");
      s->owned.push_back(s->prim_d);
    }
  } else {
    s->prim_f = dev_upload(d->prim_f32, nprim, s->owned);
    if ((flags & PHX_SNAP_F64_PRIMS) && d->prim_f64) s->prim_d = dev_upload(d->prim_f64, nprim, s->owned);
  }
  s->fmap = dev_upload(flat.data(), flat.size(), s->owned);
  s->bytes = (int64_t)(n3 * (2 * sizeof(float) + 2 * sizeof(double)) + nprim * sizeof(float) +
                       (s->prim_d ? nprim * sizeof(double) : 0) + flat.size() * sizeof(int32_t));
  ck(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "cudaStreamCreate");
  s->upload_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return s.release();
}

}  // namespace

extern "C" {

void phx_default_params(PhxRenderParams* p) {
  if (!p) return;
  std::memset(p, 0, sizeof *p);
  p->inclination = 50.0;
  p->img_width = p->img_height = 200;
  p->fov_x = p->fov_y = 40.0;
  p->r_cam = 1e4;
  p->t_init = 0.0;
  p->nfreqs = 1;
  p->frequencies[0] = 230e9;
  p->mass = 4.14e6;
  p->distance = 8.127;
  p->stepsize = 0.01;
  p->max_steps = 10000;
  p->horizon_margin = 0.01;
  p->max_order = 100;
  p->m_unit = 1e18;
  p->r_low = p->r_high = 1.0;
  p->beta_c = 1.0;
  p->sigma_cut = 1.0;
  p->thetae_min = 1e-3;
  p->thetae_max = 100.0;
  p->rt_outer = 50.0;
  p->precision = PHX_PREC_FP32;
}

int phx_snapshot_create(const PhxSnapshotDesc* desc, int32_t flags, PhxSnapshot** out) {
  return guarded([&]() -> int {
    if (!out) throw std::invalid_argument("null output handle");
    *out = create_snapshot(desc, flags);
    return PHX_OK;
  });
}

int phx_bhac_read(const char* dump_file, const char* grid_file, const PhxReadOptions* opt, int32_t flags,
                  PhxHostSnapshot** out) {
  return guarded([&]() -> int {
    if (!out || !dump_file || !grid_file) throw std::invalid_argument("null argument");
    phx::SnapshotOptions o;
    if (opt) {
      o.nspin = opt->nspin;
      o.bpol = opt->bpol;
      o.sfc = opt->sfc != 0;
      o.nlevels = opt->nlevels;
    }
    o.keep_f64 = (flags & PHX_SNAP_F64_PRIMS) != 0;
    auto hs = std::make_unique<PhxHostSnapshot>();
    hs->h = phx::load_bhac(dump_file, grid_file, o);
    for (int L = 0; L < hs->h.nlevels; L++) hs->maps.push_back(hs->h.level_map[L].data());
    *out = hs.release();
    return PHX_OK;
  });
}

int phx_bhac_describe(const PhxHostSnapshot* hs, PhxSnapshotDesc* d) {
  return guarded([&]() -> int {
    if (!hs || !d) throw std::invalid_argument("null argument");
    const phx::HostSnapshot& h = hs->h;
    std::memset(d, 0, sizeof *d);
    d->nleafs = h.nleafs;
    d->nlevels = h.nlevels;
    for (int k = 0; k < 3; k++) {
      d->nx[k] = h.nx[k];
      d->ng[k] = h.ng[k];
      d->x_lo[k] = h.x_lo[k];
      d->x_hi[k] = h.x_hi[k];
    }
    d->a = h.a;
    d->hslope = h.hslope;
    d->gam = h.gam;
    d->lb = h.lb.data();
    d->dxc = h.dxc.data();
    d->prim_f32 = h.prim_f32.data();
    d->prim_f64 = h.prim_f64.empty() ? nullptr : h.prim_f64.data();
    d->level_map = hs->maps.data();
    return PHX_OK;
  });
}

void phx_bhac_free(PhxHostSnapshot* h) { delete h; }

int phx_snapshot_load(const char* dump_file, const char* grid_file, const PhxReadOptions* opt, int32_t flags,
                      PhxSnapshot** out) {
  return guarded([&]() -> int {
    if (!out) throw std::invalid_argument("null output handle");
    if (flags & PHX_SNAP_GPU_DECODE) {
      if (!dump_file || !grid_file) throw std::invalid_argument("null argument");
      phx::SnapshotOptions o;
      if (opt) {
        o.nspin = opt->nspin;
        o.bpol = opt->bpol;
        o.sfc = opt->sfc != 0;
        o.nlevels = opt->nlevels;
      }
      const auto t0 = std::chrono::steady_clock::now();
      PhxHostSnapshot meta;
      meta.h = phx::load_bhac_meta(dump_file, grid_file, o);
      for (int L = 0; L < meta.h.nlevels; L++) meta.maps.push_back(meta.h.level_map[L].data());
      PhxSnapshotDesc d;
      phx_bhac_describe(&meta, &d);
      const double read_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      std::unique_ptr<PhxSnapshot> s(create_snapshot(&d, flags, true));
      s->decode_s = gpu_decode(s.get(), dump_file, meta.h, o.bpol);
      s->read_s = read_s;
      s->gpu_decoded = true;
      *out = s.release();
      return PHX_OK;
    }
    const auto t0 = std::chrono::steady_clock::now();
    PhxHostSnapshot* hs = nullptr;
    const int rc = phx_bhac_read(dump_file, grid_file, opt, flags, &hs);
    if (rc != PHX_OK) return rc;
    std::unique_ptr<PhxHostSnapshot> guard(hs);
    PhxSnapshotDesc d;
    phx_bhac_describe(hs, &d);
    const double read_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    *out = create_snapshot(&d, flags);
    (*out)->read_s = read_s;
    return PHX_OK;
  });
}

void phx_snapshot_destroy(PhxSnapshot* s) { delete s; }

int phx_snapshot_info(const PhxSnapshot* s, PhxSnapshotInfo* info) {
  return guarded([&]() -> int {
    if (!s || !info) throw std::invalid_argument("null argument");
    std::memset(info, 0, sizeof *info);
    info->nleafs = s->nleafs;
    info->cells = s->cells;
    info->nlevels = s->nlevels;
    for (int k = 0; k < 3; k++) {
      info->nx[k] = s->nx[k];
      info->ng[k] = s->ng[k];
      info->x_lo[k] = s->x_lo[k];
      info->x_hi[k] = s->x_hi[k];
    }
    info->a = s->a;
    info->hslope = s->hslope;
    info->gam = s->gam;
    info->has_f64_prims = s->prim_d != nullptr;
    info->gpu_decoded = s->gpu_decoded;
    info->bytes = s->bytes;
    info->read_s = s->read_s;
    info->decode_s = s->decode_s;
    info->upload_s = s->upload_s;
    return PHX_OK;
  });
}

int phx_snapshot_download(const PhxSnapshot* s, float* prim_f32, double* prim_f64) {
  return guarded([&]() -> int {
    if (!s) throw std::invalid_argument("null snapshot");
    const size_t nprim = (size_t)s->nleafs * s->cells * phx::kNPrim;
    if (prim_f32) ck(cudaMemcpy(prim_f32, s->prim_f, nprim * sizeof(float), cudaMemcpyDeviceToHost), "D2H primitives");
    if (prim_f64) {
      if (!s->prim_d) throw std::invalid_argument("the snapshot keeps no FP64 primitives");
      ck(cudaMemcpy(prim_f64, s->prim_d, nprim * sizeof(double), cudaMemcpyDeviceToHost), "D2H primitives");
    }
    return PHX_OK;
  });
}

int64_t phx_snapshot_bytes(const PhxSnapshot* s) { return s ? s->bytes : 0; }

int phx_schedule_morton(int32_t W, int32_t H, int32_t* jobs) {
  return guarded([&]() -> int {
    if (!jobs || W < 1 || H < 1 || (long long)W * H > (1LL << 31) - 1) throw std::invalid_argument("bad job list");
    std::vector<std::pair<unsigned long long, int32_t>> keyed((size_t)W * H);
    for (int i = 0; i < W; i++)
      for (int j = 0; j < H; j++) {
        unsigned long long z = 0;
        for (int b = 0; b < 16; b++)
          z |= ((unsigned long long)((i >> b) & 1) << (2 * b)) | ((unsigned long long)((j >> b) & 1) << (2 * b + 1));
        keyed[(size_t)i * H + j] = {z, i * H + j};
      }
    std::sort(keyed.begin(), keyed.end());
    for (size_t n = 0; n < keyed.size(); n++) jobs[n] = keyed[n].second;
    return PHX_OK;
  });
}

int phx_default_pixel_order(const PhxRenderParams* p) {
  if (!p) return PHX_TILE_MORTON;
  // lanes of a full grid of the single-image kernel on the current device (148 SMs x 512 if it cannot be queried)
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) !=
                                                cudaSuccess || sms < 1) {
    cudaGetLastError();
    sms = 148;
  }
  const long long lanes = (long long)sms * 512;
  return (long long)p->img_width * p->img_height <= 6 * lanes ? PHX_TILE_CENTER_4X8 : PHX_TILE_MORTON;
}

int phx_schedule_tiles(int32_t W, int32_t H, int32_t shape, int32_t* jobs) {
  if (shape == PHX_TILE_MORTON) return phx_schedule_morton(W, H, jobs);
  return guarded([&]() -> int {
    if (!jobs || W < 1 || H < 1 || (long long)W * H > (1LL << 31) - 1) throw std::invalid_argument("bad job list");
    if (shape < 0 || shape >= PHX_TILE_SHAPES) throw std::invalid_argument("unknown tile_shape");
    static const int dims[PHX_TILE_SHAPES][2] = {{8, 4}, {16, 2}, {32, 1}, {4, 8}, {2, 16}, {4, 8}};
    const int tw = dims[shape][0], th = dims[shape][1];
    const int32_t nti = (W + tw - 1) / tw, ntj = (H + th - 1) / th;
    std::vector<int32_t> tiles((size_t)nti * ntj);
    if (phx_schedule_morton(nti, ntj, tiles.data()) != PHX_OK) throw std::runtime_error(last_error());
    if (shape == PHX_TILE_CENTER_4X8) {
      // 32 x 32-pixel blocks by the distance of their centre from the image centre (in pixels), nearest first, ties
      // in Morton order; inside a block its 4 x 8 tiles in Morton order (a stable sort of the Morton tile list by
      // block rank)
      constexpr int kB = 32;
      const int32_t nbi = (W + kB - 1) / kB, nbj = (H + kB - 1) / kB;
      std::vector<int32_t> blocks((size_t)nbi * nbj), rank((size_t)nbi * nbj);
      if (phx_schedule_morton(nbi, nbj, blocks.data()) != PHX_OK) throw std::runtime_error(last_error());
      auto d2 = [&](int32_t b) {
        const int32_t bi = b / nbj, bj = b % nbj;
        const double ci = 0.5 * (bi * kB + std::min(W, (bi + 1) * kB)) - 0.5 * W;
        const double cj = 0.5 * (bj * kB + std::min(H, (bj + 1) * kB)) - 0.5 * H;
        return ci * ci + cj * cj;
      };
      std::stable_sort(blocks.begin(), blocks.end(), [&](int32_t a, int32_t b) { return d2(a) < d2(b); });
      for (size_t r = 0; r < blocks.size(); r++) rank[blocks[r]] = (int32_t)r;
      auto block_of = [&](int32_t t) {
        const int32_t ti = t / ntj, tj = t % ntj;
        return rank[(size_t)(ti * tw / kB) * nbj + tj * th / kB];
      };
      std::stable_sort(tiles.begin(), tiles.end(), [&](int32_t a, int32_t b) { return block_of(a) < block_of(b); });
    }
    size_t n = 0;
    for (const int32_t t : tiles) {
      const int32_t ti = t / ntj, tj = t % ntj;
      for (int32_t i = ti * tw; i < std::min(W, (ti + 1) * tw); i++)
        for (int32_t j = tj * th; j < std::min(H, (tj + 1) * th); j++) jobs[n++] = i * H + j;
    }
    return PHX_OK;
  });
}

int phx_render_async(PhxSnapshot* s, const PhxRenderParams* p, const int32_t* d_jobs, int64_t njobs,
                     PhxFreqOut* d_res, int32_t* d_pixstats, uint64_t* d_counters, void* stream) {
  return guarded([&]() -> int {
    if (!s || !p || !d_res || !d_counters || (njobs > 0 && !d_jobs)) throw std::invalid_argument("null argument");
    phx::check_params(*p);
    if (njobs < 0 || njobs > (int64_t)p->img_width * p->img_height) throw std::invalid_argument("njobs out of range");
    phx::LaunchShape shape;
    ck(dispatch(s, *p, d_jobs, njobs, d_res, d_pixstats, d_counters, (cudaStream_t)stream, &shape), "render launch");
    return PHX_OK;
  });
}

int phx_render(PhxSnapshot* s, const PhxRenderParams* p, const int32_t* jobs, int64_t njobs, PhxFreqOut* res,
               PhxRenderInfo* info) {
  return guarded([&]() -> int {
    if (!s || !p || !res) throw std::invalid_argument("null argument");
    phx::check_params(*p);
    const auto t0 = std::chrono::steady_clock::now();
    const int64_t npix = (int64_t)p->img_width * p->img_height;
    std::vector<int32_t> all;
    if (!jobs) {
      all.resize(npix);
      if (phx_schedule_tiles(p->img_width, p->img_height, phx_default_pixel_order(p), all.data()) != PHX_OK)
        throw std::runtime_error(last_error());
      jobs = all.data();
      njobs = npix;
    }
    if (njobs < 0 || njobs > npix) throw std::invalid_argument("njobs out of range");
    for (int64_t n = 0; n < njobs; n++)
      if (jobs[n] < 0 || jobs[n] >= npix) throw std::invalid_argument("job index out of range");
    Workspace& w = s->ws;
    const size_t nres = (size_t)npix * p->nfreqs;
    if (w.jobs_cap < (size_t)njobs) {
      cudaFree(w.jobs);
      w.jobs = nullptr;
      ck(cudaMalloc((void**)&w.jobs, std::max<size_t>(njobs, 1) * sizeof(int32_t)), "cudaMalloc jobs");
      w.jobs_cap = std::max<size_t>(njobs, 1);
    }
    if (w.res_cap < nres) {
      cudaFree(w.res);
      w.res = nullptr;
      ck(cudaMalloc((void**)&w.res, nres * sizeof(PhxFreqOut)), "cudaMalloc res");
      w.res_cap = nres;
    }
    if (!w.counters) ck(cudaMalloc((void**)&w.counters, phx::kNumCounters * sizeof(unsigned long long)), "cudaMalloc");
    if (!w.e0) ck(cudaEventCreate(&w.e0), "cudaEventCreate");
    if (!w.e1) ck(cudaEventCreate(&w.e1), "cudaEventCreate");
    cudaStream_t st = s->stream;
    ck(cudaMemcpyAsync(w.jobs, jobs, njobs * sizeof(int32_t), cudaMemcpyHostToDevice, st), "H2D jobs");
    // pixels outside the job list keep the caller's values, as in the reference (res is uploaded and read back)
    if (njobs < npix) ck(cudaMemcpyAsync(w.res, res, nres * sizeof(PhxFreqOut), cudaMemcpyHostToDevice, st), "H2D res");
    ck(cudaMemsetAsync(w.counters, 0, phx::kNumCounters * sizeof(unsigned long long), st), "memset");
    const double upload_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    phx::LaunchShape shape;
    ck(cudaEventRecord(w.e0, st), "event");
    ck(dispatch(s, *p, w.jobs, njobs, w.res, nullptr, reinterpret_cast<uint64_t*>(w.counters), st, &shape),
       "render launch");
    ck(cudaEventRecord(w.e1, st), "event");
    unsigned long long ctr[phx::kNumCounters];
    ck(cudaMemcpyAsync(res, w.res, nres * sizeof(PhxFreqOut), cudaMemcpyDeviceToHost, st), "D2H res");
    ck(cudaMemcpyAsync(ctr, w.counters, sizeof ctr, cudaMemcpyDeviceToHost, st), "D2H counters");
    ck(cudaStreamSynchronize(st), "render");
    if (info) {
      std::memset(info, 0, sizeof *info);
      std::snprintf(info->device, sizeof info->device, "%s", s->device_name);
      info->sms = s->sms;
      info->blocks = shape.grid;
      info->block = shape.block;
      info->regs = shape.regs;
      info->local_bytes = shape.local_bytes;
      float ms = 0.f;
      ck(cudaEventElapsedTime(&ms, w.e0, w.e1), "event time");
      info->kernel_s = ms * 1e-3;
      info->upload_s = upload_s;
      info->steps = (int64_t)ctr[phx::kCtrSteps];
      info->nplasma = (int64_t)ctr[phx::kCtrPlasma];
      info->bad = (int64_t)ctr[phx::kCtrBad];
      info->scans = (int64_t)ctr[phx::kCtrScans];
      info->fp64_steps = (int64_t)ctr[phx::kCtrFp64Steps];
      info->fp64_ops = (int64_t)ctr[phx::kCtrFp64Ops];
    }
    return PHX_OK;
  });
}

int phx_write_output(const PhxRenderParams* p, const PhxFreqOut* res, const char* outdir, const char* image,
                     int32_t block_size, double* flux) {
  return guarded([&]() -> int {
    if (!p || !res || !outdir || !image) throw std::invalid_argument("null argument");
    if (p->img_width < 1 || p->img_height < 1 || p->nfreqs < 1 || p->nfreqs > PHX_MAX_FREQS)
      throw std::invalid_argument("bad image size or frequency count");
    const std::string mode = image, dir = outdir;
    if (mode != "hdf5" && mode != "text" && mode != "both" && mode != "none")
      throw std::invalid_argument("image must be hdf5, text, both or none");
    const std::vector<PhxFreqOut> r(res, res + (size_t)p->img_width * p->img_height * p->nfreqs);
    bool want_text = mode == "text" || mode == "both";
    if (mode == "hdf5" || mode == "both") {
      std::string err;
      if (!phx::write_image_hdf5(dir + "/img_data.h5", *p, block_size, r, &err)) want_text = true;
    }
    if (want_text)
      for (int f = 0; f < p->nfreqs; f++) {
        const std::string ip = dir + "/image" + (p->nfreqs == 1 ? "" : "_" + std::to_string(f)) + ".dat";
        if (!phx::write_image_text(ip, *p, r, f)) throw std::runtime_error("cannot write " + ip);
      }
    if (!phx::write_spectrum(dir + "/spectrum.dat", *p, r)) throw std::runtime_error("cannot write spectrum.dat");
    if (flux)
      for (int f = 0; f < p->nfreqs; f++) phx::compute_spec(*p, r, f, flux + 4 * f);
    return PHX_OK;
  });
}

const char* phx_last_error(void) { return last_error().c_str(); }

const char* phx_version(void) { return "phoenix-b200 0.1 (sm_100a)"; }

}  // extern "C"

// ---------------------------------------------------------------------------------------------------------------
// Rendering without any device allocation.
//
// Some callers cannot call cudaMalloc: a host application that owns all device memory through its own pool or arena
// (so a library allocation would fragment it or fail its accounting), or a serving loop that must not let an
// allocation synchronize the device and stall the other streams in flight.  phx_render_noalloc serves them: the
// job list and the kernel's scratch (work-queue head and counter block) live in the fixed array below, which the
// library's module holds on every GPU that loads it, until the process exits.  The caller passes the snapshot,
// the parameters, the job list in host memory and the device result buffer; nothing else is allocated.
//
// Layout of the array: [0, 256) the 16-word counter block (word 0 = queue head), [256, 256 + 4 * kNoAllocMaxJobs)
// the job list.  Every call shares it and it keeps the last call's contents: the counter block is cleared on the
// stream before each launch, and calls that overlap on the GPU race on it.
namespace {

constexpr size_t kNoAllocHeader = 256;
constexpr int64_t kNoAllocMaxJobs = PHX_NOALLOC_MAX_JOBS;
constexpr size_t kNoAllocBytes = kNoAllocHeader + sizeof(int32_t) * (size_t)kNoAllocMaxJobs;
static_assert(phx::kNumCounters * sizeof(unsigned long long) <= kNoAllocHeader, "counter block must fit the header");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
void* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of the scratch array on the current device, resolved once per device (the symbol's host-side name
// is only a stand-in and must never be passed to a kernel).  Kept until the process exits: a cudaDeviceReset would
// unload the module and leave it stale, so the entry point is not for use across a device reset.
void* noalloc_scratch(int device) {
  if (device < 0 || device >= kNoAllocMaxDevices) throw std::invalid_argument("device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[device]) {
    void* ptr = nullptr;
    ck(cudaGetSymbolAddress(&ptr, g_noalloc_scratch), "cudaGetSymbolAddress");
    g_noalloc_ptr[device] = ptr;
  }
  return g_noalloc_ptr[device];
}

}  // namespace

extern "C" int phx_render_noalloc(PhxSnapshot* s, const PhxRenderParams* p, const int32_t* jobs, int64_t njobs,
                                  PhxFreqOut* d_res, void* stream) {
  return guarded([&]() -> int {
    if (!s || !p || !d_res || (njobs > 0 && !jobs)) throw std::invalid_argument("null argument");
    phx::check_params(*p);
    if (njobs < 0) throw std::invalid_argument("njobs must be >= 0");
    if (njobs > kNoAllocMaxJobs)
      throw std::invalid_argument("njobs = " + std::to_string(njobs) + " exceeds the no-allocation limit of " +
                                  std::to_string(kNoAllocMaxJobs) + " jobs (PHX_NOALLOC_MAX_JOBS)");
    const int64_t npix = (int64_t)p->img_width * p->img_height;
    for (int64_t n = 0; n < njobs; n++)
      if (jobs[n] < 0 || jobs[n] >= npix) throw std::invalid_argument("job index out of range");
    int device = 0;
    ck(cudaGetDevice(&device), "cudaGetDevice");
    if (device != s->device) throw std::invalid_argument("the snapshot lives on another device");
    unsigned char* base = static_cast<unsigned char*>(noalloc_scratch(device));
    uint64_t* counters = reinterpret_cast<uint64_t*>(base);
    int32_t* d_jobs = reinterpret_cast<int32_t*>(base + kNoAllocHeader);
    cudaStream_t st = (cudaStream_t)stream;
    ck(cudaMemsetAsync(counters, 0, phx::kNumCounters * sizeof(unsigned long long), st), "memset scratch");
    if (njobs > 0) ck(cudaMemcpyAsync(d_jobs, jobs, njobs * sizeof(int32_t), cudaMemcpyHostToDevice, st), "H2D jobs");
    phx::LaunchShape shape;
    ck(dispatch(s, *p, d_jobs, njobs, d_res, nullptr, counters, st, &shape), "render launch");
    return PHX_OK;
  });
}
