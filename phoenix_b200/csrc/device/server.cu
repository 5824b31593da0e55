// The served render loop: continuous batching of render requests into one running queue kernel.
//
// A server keeps snapshots resident and owns a device arena for request results and job lists.  Requests are
// admitted first-in first-out while their footprint (results + job list) fits the arena and an item slot is free.  An
// admitted request is published into the running queue kernel (queue.cuh) without stopping it: its item descriptor and
// tiles are copied on a control stream, then the queue tail; lanes that finished earlier rays pick its rays up at
// their next refill point, so requests that arrive while others are on the GPU share the device with them.  The
// kernel's last lane of a request raises the request's completion word in host-mapped memory; the scheduler thread
// then copies the result back, frees its arena space and admits more.
//
// Generations.  Item slots and tile positions are used once per run of the kernel ("generation"): a descriptor is
// never rewritten while a kernel that may have cached it runs.  When the server has been idle for `linger_ms`, or a
// generation's item slots or tiles run out, the scheduler lets the in-flight requests finish, sets the stop word,
// waits for the kernel to leave, resets the queue and starts the next generation at the next admission.
//
// All CUDA work of a server happens on its scheduler thread; the API calls only exchange records with it.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "internal.hpp"
#include "queue.cuh"

using namespace phx_capi;

namespace {

using Clock = std::chrono::steady_clock;

double seconds_since(Clock::time_point t0) {
  return std::chrono::duration<double>(Clock::now() - t0).count();
}

// First-fit allocator over [0, size) with coalescing (offsets and sizes in 256-byte units of the arena).
class ArenaAlloc {
 public:
  explicit ArenaAlloc(size_t size) : size_(size) {
    if (size) free_[0] = size;
  }
  bool alloc(size_t n, size_t* off) {
    n = (n + 255) & ~(size_t)255;
    for (auto it = free_.begin(); it != free_.end(); ++it)
      if (it->second >= n) {
        *off = it->first;
        const size_t rest = it->second - n, start = it->first + n;
        free_.erase(it);
        if (rest) free_[start] = rest;
        used_ += n;
        return true;
      }
    return false;
  }
  void release(size_t off, size_t n) {
    n = (n + 255) & ~(size_t)255;
    used_ -= n;
    auto it = free_.emplace(off, n).first;
    auto next = std::next(it);
    if (next != free_.end() && it->first + it->second == next->first) {
      it->second += next->second;
      free_.erase(next);
    }
    if (it != free_.begin()) {
      auto prev = std::prev(it);
      if (prev->first + prev->second == it->first) {
        prev->second += it->second;
        free_.erase(it);
      }
    }
  }
  size_t used() const { return used_; }

 private:
  size_t size_, used_ = 0;
  std::map<size_t, size_t> free_;
};

struct Request {
  int64_t id = 0;
  int32_t snap = 0;
  PhxRenderParams p{};
  int32_t state = PHX_REQ_QUEUED;
  int32_t slot = -1;
  size_t out_off = 0, out_bytes = 0;
  int64_t rays = 0;
  int64_t ntiles = 0, next_tile = 0;  // tiles of the request, and the first one not yet published
  int retries = 0;                     // times it went back to the queue after the kernel ended early
  std::vector<PhxFreqOut> host;
  PhxRequestTiming t{};
  Clock::time_point submitted;
  std::string error;
};

}  // namespace

struct PhxServer {
  PhxServerOptions o{};
  int device = 0, sms = 0;
  int nf_slots = 4;
  std::vector<PhxSnapshot*> snaps;
  // device state
  unsigned char* arena = nullptr;
  std::unique_ptr<ArenaAlloc> alloc;
  void* items = nullptr;  // max_items descriptors
  size_t item_bytes = 0;
  phx::TileDesc* tiles = nullptr;
  unsigned long long* item_ctr = nullptr;
  unsigned long long* ctl = nullptr;
  unsigned long long* counters = nullptr;
  int32_t* done_host = nullptr;  // host-mapped completion words
  int32_t* done_dev = nullptr;
  unsigned char* staging = nullptr;  // pinned: one descriptor + a request's tiles + the tail word
  size_t staging_bytes = 0;
  std::map<std::tuple<int32_t, int32_t, int>, size_t> job_tables;  // job list per (size, pixel order): arena offset
  cudaStream_t compute = nullptr, control = nullptr, copy = nullptr;
  cudaEvent_t kernel_done = nullptr;
  // writes request r's item descriptor into dst (sizeof descriptor bytes)
  std::function<void(const Request&, const int32_t* jobs, unsigned char* dst)> write_item;
  std::function<cudaError_t(cudaStream_t, phx::LaunchShape*)> launch;
  // generation
  bool kernel_running = false;
  int32_t next_slot = 0;
  unsigned long long tiles_published = 0;
  unsigned long long tiles_reserved = 0;  // published + not yet published tiles of the admitted requests
  std::vector<int64_t> unpublished;       // admitted requests with tiles left to publish, in admission order
  unsigned long long* head_host = nullptr;  // pinned: the queue head read back each tick
  Clock::time_point idle_since;
  int64_t generations = 0;
  phx::LaunchShape lshape{};
  // requests
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<int64_t> pending;
  std::unordered_map<int64_t, std::unique_ptr<Request>> reqs;
  std::vector<int64_t> slot_req;
  int64_t next_id = 1;
  int64_t inflight = 0;
  bool shutdown = false;
  std::string fatal;
  Clock::time_point t0 = Clock::now();
  PhxServerStats stats{};
  std::thread worker;

  ~PhxServer();
  void run();
  void tick();
  bool admit_one(Request& r);
  void start_generation();
  void stop_kernel();
  void reap();
  void fail_inflight(const std::string& why);
  void requeue_inflight();
  void publish();
  void ensure_kernel();
  void reset_queue();
};

namespace {

template <phx::Mode M, class PT>
void bind_mode(PhxServer* s) {
  using R = typename phx::Policy<M>::R;
  using Item = phx::ItemDesc<R, PT>;
  s->item_bytes = sizeof(Item);
  PhxServer* self = s;
  s->write_item = [self](const Request& r, const int32_t* jobs, unsigned char* dst) {
    Item it;
    std::memset((void*)&it, 0, sizeof it);
    const PhxSnapshot* sn = self->snaps[r.snap];
    it.rc = phx::make_consts<R>(r.p, sn->a, sn->hslope);
    it.snap = view_for<M, PT>(sn);
    it.snap_d = it.snap.fp64_view();
    it.jobs = jobs;
    it.out = reinterpret_cast<double*>(self->arena + r.out_off);
    it.pixstats = nullptr;
    it.ctr = self->item_ctr + (size_t)phx::kItemCounters * r.slot;
    it.nrays = (unsigned long long)r.rays;
    it.done = self->done_dev + r.slot;
    std::memcpy(dst, &it, sizeof it);
  };
  s->launch = [self](cudaStream_t st, phx::LaunchShape* ls) {
    phx::QueueArgs<R, PT> A;
    A.items = reinterpret_cast<const Item*>(self->items);
    A.tiles = self->tiles;
    A.ctl = self->ctl;
    A.counters = self->counters;
    A.tile_mask = (unsigned)(self->o.max_tiles - 1);
    A.tile_rays = self->o.tile_rays;
    A.period = self->o.period;
    A.idle_ns = self->o.idle_ns;
    A.idle_limit = self->o.idle_limit;
    phx::QueueShape q{self->o.blocks_per_sm, self->o.period, self->o.refill_lanes};
    return phx::launch_queue<M, PT>(A, self->nf_slots, self->sms, q, 0, st, ls);
  };
}

}  // namespace

PhxServer::~PhxServer() {
  {
    std::lock_guard<std::mutex> lk(mu);
    shutdown = true;
  }
  cv_work.notify_all();
  if (worker.joinable()) worker.join();
  if (kernel_done) cudaEventDestroy(kernel_done);
  for (cudaStream_t st : {compute, control, copy})
    if (st) cudaStreamDestroy(st);
  cudaFree(arena);
  cudaFree(items);
  cudaFree(tiles);
  cudaFree(item_ctr);
  cudaFree(ctl);
  cudaFree(counters);
  if (done_host) cudaFreeHost(done_host);
  if (head_host) cudaFreeHost(head_host);
  if (staging) cudaFreeHost(staging);
}

// Resets the queue for a new generation (no kernel is running).
void PhxServer::start_generation() {
  ck(cudaMemsetAsync(ctl, 0, phx::kQWords * sizeof(unsigned long long), control), "reset queue");
  ck(cudaMemsetAsync(item_ctr, 0, (size_t)phx::kItemCounters * o.max_items * sizeof(unsigned long long), control),
     "reset item counters");
  ck(cudaStreamSynchronize(control), "reset queue");
  std::memset(done_host, 0, sizeof(int32_t) * o.max_items);
  reset_queue();
  std::fill(slot_req.begin(), slot_req.end(), 0);
}

// Stops the running kernel (called with nothing in flight).  A kernel that already left by its bounded idle wait
// (status word set) is not an error here: no request was lost, and the next admission starts a new generation.
void PhxServer::stop_kernel() {
  if (!kernel_running) return;
  unsigned long long* one = reinterpret_cast<unsigned long long*>(staging);
  *one = 1ull;
  ck(cudaMemcpyAsync(ctl + phx::kQStop, one, sizeof *one, cudaMemcpyHostToDevice, control), "stop word");
  ck(cudaStreamSynchronize(control), "stop word");
  ck(cudaStreamSynchronize(compute), "queue kernel");
  kernel_running = false;
  unsigned long long status = 0;
  ck(cudaMemcpy(&status, ctl + phx::kQStatus, sizeof status, cudaMemcpyDeviceToHost), "status word");
  if (status) {
    std::lock_guard<std::mutex> lk(mu);
    stats.idle_exits++;
  }
}

// Admits request r if its footprint fits and the generation has room; publishes it into the queue.
bool PhxServer::admit_one(Request& r) {
  const int64_t npix = (int64_t)r.p.img_width * r.p.img_height;
  const int64_t ntiles = (npix + o.tile_rays - 1) / o.tile_rays;
  if (next_slot >= o.max_items || (long long)(tiles_reserved + ntiles) > o.max_tiles) return false;
  const int order = phx_default_pixel_order(&r.p);
  const auto key = std::make_tuple(r.p.img_width, r.p.img_height, order);
  size_t jobs_off = 0;
  auto jt = job_tables.find(key);
  if (jt == job_tables.end()) {
    if (!alloc->alloc((size_t)npix * sizeof(int32_t), &jobs_off)) return false;
    std::vector<int32_t> m((size_t)npix);
    if (phx_schedule_tiles(r.p.img_width, r.p.img_height, order, m.data()) != PHX_OK)
      throw std::runtime_error(last_error());
    ck(cudaMemcpyAsync(arena + jobs_off, m.data(), m.size() * sizeof(int32_t), cudaMemcpyHostToDevice, control),
       "H2D jobs");
    ck(cudaStreamSynchronize(control), "H2D jobs");
    job_tables[key] = jobs_off;
    stats.job_table_bytes += (int64_t)(npix * sizeof(int32_t));
  } else {
    jobs_off = jt->second;
  }
  r.out_bytes = (size_t)npix * r.p.nfreqs * sizeof(PhxFreqOut);
  if (!alloc->alloc(r.out_bytes, &r.out_off)) return false;
  if (!kernel_running && next_slot == 0 && tiles_reserved == 0) start_generation();
  r.slot = next_slot++;
  r.rays = npix;
  r.ntiles = ntiles;
  r.next_tile = 0;
  tiles_reserved += ntiles;
  slot_req[r.slot] = r.id;
  // the descriptor goes in now; its tiles are published by publish() as the queue drains
  write_item(r, reinterpret_cast<const int32_t*>(arena + jobs_off), staging);
  ck(cudaMemcpyAsync(static_cast<unsigned char*>(items) + item_bytes * r.slot, staging, item_bytes,
                     cudaMemcpyHostToDevice, control),
     "H2D item");
  ck(cudaStreamSynchronize(control), "H2D item");
  unpublished.push_back(r.id);
  {
    std::lock_guard<std::mutex> lk(mu);
    r.state = PHX_REQ_RUNNING;
    r.t.admitted_s = seconds_since(r.submitted);
    inflight++;
  }
  return true;
}

// Starts the generation's kernel once it has published work: a kernel launched onto an empty queue would spend its
// bounded idle wait before the first tiles arrive.
void PhxServer::ensure_kernel() {
  if (kernel_running || tiles_published == 0) return;
  ck(launch(compute, &lshape), "queue kernel launch");
  ck(cudaEventRecord(kernel_done, compute), "event");
  kernel_running = true;
  generations++;
}

// Publishes tiles of the admitted requests.  Small requests (at most small_rays rays) go in whole as soon as they are
// admitted; large ones go in first in, first out, a chunk at a time while the queue's backlog of published but
// unclaimed rays is below half a grid-load of lanes (about 20 ms of work on a B200: far more than one scheduler tick
// needs to top it up, and little for a later request to wait behind).  A small request that arrives behind a large
// one therefore waits for that backlog, not for every ray of the large one, while the large ones keep their order and
// their rays' coherence (interleaving them all round robin mixes snapshots and images in the caches and costs
// throughput).
void PhxServer::publish() {
  if (unpublished.empty()) return;
  ck(cudaMemcpyAsync(head_host, ctl + phx::kQHead, sizeof *head_host, cudaMemcpyDeviceToHost, copy), "D2H head");
  ck(cudaStreamSynchronize(copy), "D2H head");
  const long long slots = (long long)tiles_published * o.tile_rays;
  long long backlog = slots - (long long)*head_host;  // idle lanes' claims can pass the tail: then nothing is left
  if (backlog < 0) backlog = 0;
  // resident lanes of the running kernel (before the generation's first launch: a whole-SM block of 512 per SM)
  const long long lanes = lshape.grid > 0 ? (long long)lshape.grid * lshape.block : (long long)sms * 512;
  const long long limit = o.backlog_rays > 0 ? o.backlog_rays : lanes / 2;
  phx::TileDesc* td = reinterpret_cast<phx::TileDesc*>(staging + ((item_bytes + 255) & ~(size_t)255));
  int64_t n = 0;
  auto put = [&](Request* r, int64_t m) {
    for (int64_t t = r->next_tile; t < r->next_tile + m; t++)
      td[n++] = {r->slot, (int32_t)(t * o.tile_rays), (int32_t)std::min<int64_t>(o.tile_rays, r->rays - t * o.tile_rays),
                 0};
    r->next_tile += m;
  };
  std::vector<int64_t> keep;
  std::vector<Request*> large;
  {
    std::lock_guard<std::mutex> lk(mu);
    for (int64_t id : unpublished) {
      Request* r = reqs.at(id).get();
      if (r->rays <= o.small_rays) put(r, r->ntiles - r->next_tile);
      else large.push_back(r);
    }
  }
  for (Request* r : large) {
    while (r->next_tile < r->ntiles && backlog + n * o.tile_rays < limit)
      put(r, std::min<int64_t>(o.publish_chunk, r->ntiles - r->next_tile));
    if (r->next_tile < r->ntiles) keep.push_back(r->id);
  }
  unpublished.swap(keep);
  if (n == 0) return;
  // tiles, then the tail: in this order on the control stream
  ck(cudaMemcpyAsync(tiles + tiles_published, td, n * sizeof(phx::TileDesc), cudaMemcpyHostToDevice, control),
     "H2D tiles");
  tiles_published += n;
  unsigned long long* tail = reinterpret_cast<unsigned long long*>(staging + staging_bytes - 256);
  *tail = tiles_published;
  ck(cudaMemcpyAsync(ctl + phx::kQTail, tail, sizeof *tail, cudaMemcpyHostToDevice, control), "H2D tail");
  ck(cudaStreamSynchronize(control), "publish");
}

// A new generation starts at the next admission (no kernel is running).
void PhxServer::reset_queue() {
  next_slot = 0;
  tiles_published = 0;
  tiles_reserved = 0;
  unpublished.clear();
}

// Completed requests: copy results back, free their arena space.
void PhxServer::reap() {
  for (int32_t s = 0; s < next_slot; s++) {
    const int64_t id = slot_req[s];
    if (!id) continue;
    if (!reinterpret_cast<volatile int32_t*>(done_host)[s]) continue;
    Request* r;
    {
      std::lock_guard<std::mutex> lk(mu);
      r = reqs.at(id).get();
    }
    r->host.resize((size_t)r->rays * r->p.nfreqs);
    ck(cudaMemcpyAsync(r->host.data(), arena + r->out_off, r->out_bytes, cudaMemcpyDeviceToHost, copy), "D2H results");
    unsigned long long c[phx::kItemCounters];
    ck(cudaMemcpyAsync(c, item_ctr + (size_t)phx::kItemCounters * s, sizeof c, cudaMemcpyDeviceToHost, copy),
       "D2H counters");
    ck(cudaStreamSynchronize(copy), "D2H results");
    alloc->release(r->out_off, r->out_bytes);
    slot_req[s] = 0;
    r->t.steps = (int64_t)c[phx::kItSteps];
    r->t.nplasma = (int64_t)c[phx::kItPlasma];
    r->t.bad = (int64_t)c[phx::kItBad];
    r->t.rays = r->rays;
    {
      std::lock_guard<std::mutex> lk(mu);
      r->t.done_s = seconds_since(r->submitted);
      r->state = PHX_REQ_DONE;
      inflight--;
      stats.completed++;
      stats.rays += r->rays;
      stats.steps += r->t.steps;
    }
    cv_done.notify_all();
  }
}

// Fails every request in flight (the kernel left early) and resets the queue.
void PhxServer::fail_inflight(const std::string& why) {
  std::lock_guard<std::mutex> lk(mu);
  for (int32_t sl = 0; sl < next_slot; sl++) {
    const int64_t id = slot_req[sl];
    if (!id) continue;
    Request* r = reqs.at(id).get();
    alloc->release(r->out_off, r->out_bytes);
    r->state = PHX_REQ_FAILED;
    r->error = why;
    slot_req[sl] = 0;
    inflight--;
  }
  reset_queue();
  cv_done.notify_all();
}

// The kernel left by its bounded idle wait while requests were in flight (idle warps give up after idle_limit polls;
// one that gave up holding a claim past the tail leaves that slot unserved).  Their results are incomplete: each goes
// back to the front of the queue, in admission order, to be rendered again from scratch in a new generation (every
// pixel is written once per run), at most kMaxRetries times before it fails.
void PhxServer::requeue_inflight() {
  constexpr int kMaxRetries = 2;
  std::lock_guard<std::mutex> lk(mu);
  std::vector<int64_t> back;
  for (int32_t sl = 0; sl < next_slot; sl++) {
    const int64_t id = slot_req[sl];
    if (!id) continue;
    Request* r = reqs.at(id).get();
    alloc->release(r->out_off, r->out_bytes);
    slot_req[sl] = 0;
    inflight--;
    if (r->retries < kMaxRetries) {
      r->retries++;
      r->state = PHX_REQ_QUEUED;
      stats.retries++;
      back.push_back(id);
    } else {
      r->state = PHX_REQ_FAILED;
      r->error = "the queue kernel kept leaving before finishing the request (idle limit reached)";
    }
  }
  pending.insert(pending.begin(), back.begin(), back.end());
  reset_queue();
  cv_done.notify_all();
}

void PhxServer::tick() {
  reap();
  if (kernel_running && cudaEventQuery(kernel_done) == cudaSuccess) {
    // the kernel left without being stopped: only its bounded idle wait does that
    kernel_running = false;
    bool any;
    {
      std::lock_guard<std::mutex> lk(mu);
      any = inflight > 0;
      stats.idle_exits++;
    }
    reap();
    if (any) requeue_inflight();
    reset_queue();
  }
  const bool fresh = !kernel_running && next_slot == 0 && tiles_reserved == 0;
  // admissions, first in first out
  bool head_rejected = false;
  for (;;) {
    Request* r = nullptr;
    {
      std::lock_guard<std::mutex> lk(mu);
      if (pending.empty()) break;
      r = reqs.at(pending.front()).get();
    }
    if (!admit_one(*r)) {
      head_rejected = true;
      break;
    }
    std::lock_guard<std::mutex> lk(mu);
    pending.pop_front();
  }
  publish();
  ensure_kernel();
  int64_t nin;
  bool has_pending;
  {
    std::lock_guard<std::mutex> lk(mu);
    nin = inflight;
    has_pending = !pending.empty();
  }
  if (head_rejected && nin == 0 && fresh) {
    // nothing in flight, a fresh generation, and the head request still does not fit: it never will
    std::lock_guard<std::mutex> lk(mu);
    Request* r = reqs.at(pending.front()).get();
    pending.pop_front();
    r->state = PHX_REQ_FAILED;
    r->error = "request does not fit the server's arena or queue";
    cv_done.notify_all();
    return;
  }
  if (nin > 0 || has_pending) idle_since = Clock::now();
  if (kernel_running && nin == 0) {
    // the generation is exhausted (the head request does not fit), or the server has idled long enough
    const double idle_ms = std::chrono::duration<double, std::milli>(Clock::now() - idle_since).count();
    if (head_rejected || (!has_pending && idle_ms >= o.linger_ms)) {
      stop_kernel();
      reset_queue();
    }
  }
}

void PhxServer::run() {
  try {
    ck(cudaSetDevice(device), "cudaSetDevice");
    idle_since = Clock::now();
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu);
        if (shutdown) break;
        if (pending.empty() && inflight == 0 && !kernel_running)
          cv_work.wait_for(lk, std::chrono::milliseconds(50));
        if (shutdown) break;
      }
      tick();
      if (kernel_running) std::this_thread::sleep_for(std::chrono::microseconds(o.poll_us));
    }
    // drain: let in-flight requests finish (or the kernel leave), then stop the kernel
    for (;;) {
      reap();
      {
        std::lock_guard<std::mutex> lk(mu);
        if (inflight == 0) break;
      }
      if (!kernel_running || cudaEventQuery(kernel_done) == cudaSuccess) {
        kernel_running = false;
        reap();
        fail_inflight("server shut down");
        break;
      }
      std::this_thread::sleep_for(std::chrono::microseconds(o.poll_us));
    }
    stop_kernel();
  } catch (const std::exception& e) {
    std::lock_guard<std::mutex> lk(mu);
    fatal = e.what();
    for (auto& kv : reqs)
      if (kv.second->state == PHX_REQ_QUEUED || kv.second->state == PHX_REQ_RUNNING) {
        kv.second->state = PHX_REQ_FAILED;
        kv.second->error = fatal;
      }
    cv_done.notify_all();
    if (kernel_running) {
      unsigned long long one = 1;
      cudaMemcpy(ctl + phx::kQStop, &one, sizeof one, cudaMemcpyHostToDevice);
      cudaStreamSynchronize(compute);
      kernel_running = false;
    }
  }
}

namespace {

PhxServer* create_server(PhxSnapshot* const* snaps, int32_t nsnaps, const PhxServerOptions* opt) {
  if (!snaps || nsnaps < 1) throw std::invalid_argument("a server needs at least one snapshot");
  auto s = std::make_unique<PhxServer>();
  phx_default_server_options(&s->o);
  if (opt) s->o = *opt;
  PhxServerOptions& o = s->o;
  if (o.tile_rays <= 0) o.tile_rays = 32;
  if (o.max_items <= 0) o.max_items = 4096;
  if (o.max_tiles <= 0) o.max_tiles = 1 << 22;
  if ((o.max_tiles & (o.max_tiles - 1)) != 0) throw std::invalid_argument("max_tiles must be a power of two");
  if (o.max_freqs <= 0) o.max_freqs = 4;
  if (o.max_freqs > 4 && o.precision != PHX_PREC_FP32) throw std::invalid_argument("more than 4 frequencies: FP32 only");
  if (o.period <= 0) o.period = phx::kDefaultQueuePeriod;
  if (o.refill_lanes < 0 || o.refill_lanes > 32) throw std::invalid_argument("refill_lanes must be in 0..32");
  if (o.refill_lanes == 0) o.refill_lanes = 32;
  if (o.idle_ns <= 0) o.idle_ns = 2000;
  if (o.idle_limit <= 0) o.idle_limit = 5000000;
  if (o.linger_ms < 0) o.linger_ms = 0;
  if (o.poll_us <= 0) o.poll_us = 50;
  if (o.publish_chunk <= 0) o.publish_chunk = 64;
  if (o.small_rays < 0) o.small_rays = 0;
  if (o.precision < PHX_PREC_FP32 || o.precision > PHX_PREC_MIXED) throw std::invalid_argument("unknown precision");
  ck(cudaGetDevice(&s->device), "cudaGetDevice");
  int64_t snap_bytes = 0;
  bool f64prims = true;
  for (int32_t i = 0; i < nsnaps; i++) {
    if (!snaps[i]) throw std::invalid_argument("null snapshot");
    if (snaps[i]->device != s->device) throw std::invalid_argument("every snapshot must live on the current device");
    s->snaps.push_back(snaps[i]);
    snap_bytes += snaps[i]->bytes;
    f64prims = f64prims && snaps[i]->prim_d;
    s->sms = snaps[i]->sms;
  }
  s->nf_slots = o.max_freqs <= 1 ? 1 : o.max_freqs <= 4 ? 4 : phx::kMaxFreqs;
  switch (o.precision) {
    case PHX_PREC_FP32: bind_mode<phx::Mode::kFP32, float>(s.get()); break;
    case PHX_PREC_MIXED: bind_mode<phx::Mode::kMixed, float>(s.get()); break;
    default:
      if (f64prims) bind_mode<phx::Mode::kFP64, double>(s.get());
      else bind_mode<phx::Mode::kFP64, float>(s.get());
  }
  const int64_t tables = (int64_t)s->item_bytes * o.max_items + (int64_t)sizeof(phx::TileDesc) * o.max_tiles +
                         (int64_t)sizeof(unsigned long long) * (phx::kItemCounters * (int64_t)o.max_items + 64);
  int64_t arena = o.arena_bytes;
  if (arena <= 0) arena = std::min<int64_t>(o.memory_budget - snap_bytes - tables, (int64_t)16 << 30);
  if (o.memory_budget > 0 && snap_bytes + tables + arena > o.memory_budget)
    throw std::invalid_argument("snapshots, queue tables and arena exceed the memory budget");
  if (arena < (1 << 20)) throw std::invalid_argument("no room for a result arena within the memory budget");
  ck(cudaMalloc((void**)&s->arena, (size_t)arena), "cudaMalloc arena");
  s->alloc = std::make_unique<ArenaAlloc>((size_t)arena);
  ck(cudaMalloc(&s->items, s->item_bytes * o.max_items), "cudaMalloc items");
  ck(cudaMalloc((void**)&s->tiles, sizeof(phx::TileDesc) * o.max_tiles), "cudaMalloc tiles");
  ck(cudaMalloc((void**)&s->item_ctr, sizeof(unsigned long long) * phx::kItemCounters * o.max_items), "cudaMalloc");
  ck(cudaMalloc((void**)&s->ctl, sizeof(unsigned long long) * phx::kQWords), "cudaMalloc");
  ck(cudaMalloc((void**)&s->counters, sizeof(unsigned long long) * phx::kNumCounters), "cudaMalloc");
  ck(cudaMemset(s->counters, 0, sizeof(unsigned long long) * phx::kNumCounters), "memset");
  ck(cudaHostAlloc((void**)&s->done_host, sizeof(int32_t) * o.max_items, cudaHostAllocMapped), "cudaHostAlloc");
  ck(cudaHostGetDevicePointer((void**)&s->done_dev, s->done_host, 0), "cudaHostGetDevicePointer");
  ck(cudaHostAlloc((void**)&s->head_host, sizeof(unsigned long long), cudaHostAllocDefault), "cudaHostAlloc");
  // staging: descriptor | tiles of the largest request that fits the queue | tail word
  s->staging_bytes = ((s->item_bytes + 255) & ~(size_t)255) + sizeof(phx::TileDesc) * (size_t)o.max_tiles + 256;
  ck(cudaHostAlloc((void**)&s->staging, s->staging_bytes, cudaHostAllocDefault), "cudaHostAlloc staging");
  ck(cudaStreamCreateWithFlags(&s->compute, cudaStreamNonBlocking), "cudaStreamCreate");
  ck(cudaStreamCreateWithFlags(&s->control, cudaStreamNonBlocking), "cudaStreamCreate");
  ck(cudaStreamCreateWithFlags(&s->copy, cudaStreamNonBlocking), "cudaStreamCreate");
  ck(cudaEventCreateWithFlags(&s->kernel_done, cudaEventDisableTiming), "cudaEventCreate");
  s->slot_req.assign(o.max_items, 0);
  s->stats.arena_bytes = arena;
  s->stats.snapshot_bytes = snap_bytes;
  s->stats.table_bytes = tables;
  s->start_generation();
  PhxServer* raw = s.get();
  s->worker = std::thread([raw] { raw->run(); });
  return s.release();
}

}  // namespace

extern "C" {

void phx_default_server_options(PhxServerOptions* o) {
  if (!o) return;
  std::memset(o, 0, sizeof *o);
  o->memory_budget = (int64_t)150 << 30;
  o->precision = PHX_PREC_FP32;
  o->max_freqs = 4;
  o->tile_rays = 32;
  o->period = phx::kDefaultQueuePeriod;
  o->refill_lanes = 32;
  o->blocks_per_sm = 0;
  o->max_items = 4096;
  o->max_tiles = 1 << 22;
  o->idle_ns = 2000;
  o->idle_limit = 5000000;
  o->linger_ms = 20.0;
  o->poll_us = 50;
  o->publish_chunk = 64;
  o->backlog_rays = 0;
  o->small_rays = 65536;
}

int phx_server_create(PhxSnapshot* const* snaps, int32_t nsnaps, const PhxServerOptions* opt, PhxServer** out) {
  return guarded([&]() -> int {
    if (!out) throw std::invalid_argument("null output handle");
    *out = create_server(snaps, nsnaps, opt);
    return PHX_OK;
  });
}

int phx_server_submit(PhxServer* s, int32_t snapshot, const PhxRenderParams* p, int64_t* request) {
  return guarded([&]() -> int {
    if (!s || !p || !request) throw std::invalid_argument("null argument");
    if (snapshot < 0 || snapshot >= (int32_t)s->snaps.size()) throw std::invalid_argument("snapshot id out of range");
    phx::check_params(*p);
    if (p->precision != s->o.precision) throw std::invalid_argument("request precision differs from the server's");
    if (p->nfreqs > s->nf_slots) throw std::invalid_argument("request has more frequencies than the server's slots");
    auto r = std::make_unique<Request>();
    r->snap = snapshot;
    r->p = *p;
    r->submitted = Clock::now();
    {
      std::lock_guard<std::mutex> lk(s->mu);
      if (!s->fatal.empty()) throw std::runtime_error("server failed: " + s->fatal);
      r->id = s->next_id++;
      r->t.submitted_s = std::chrono::duration<double>(r->submitted - s->t0).count();
      *request = r->id;
      s->pending.push_back(r->id);
      s->reqs[r->id] = std::move(r);
      s->stats.submitted++;
    }
    s->cv_work.notify_all();
    return PHX_OK;
  });
}

int phx_server_poll(PhxServer* s, int64_t request, int32_t* state) {
  return guarded([&]() -> int {
    if (!s || !state) throw std::invalid_argument("null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(request);
    if (it == s->reqs.end()) throw std::invalid_argument("unknown request");
    *state = it->second->state;
    return PHX_OK;
  });
}

int phx_server_wait(PhxServer* s, int64_t request, double timeout_s, int32_t* state) {
  return guarded([&]() -> int {
    if (!s) throw std::invalid_argument("null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(request);
    if (it == s->reqs.end()) throw std::invalid_argument("unknown request");
    Request* r = it->second.get();
    const auto until = Clock::now() + std::chrono::duration<double>(timeout_s > 0 ? timeout_s : 1e9);
    s->cv_done.wait_until(lk, until, [&] { return r->state == PHX_REQ_DONE || r->state == PHX_REQ_FAILED; });
    if (state) *state = r->state;
    if (r->state == PHX_REQ_FAILED) throw std::runtime_error(r->error);
    if (r->state != PHX_REQ_DONE) return fail(PHX_E_TIMEOUT, "request not finished within the timeout");
    return PHX_OK;
  });
}

int phx_server_result(PhxServer* s, int64_t request, PhxFreqOut* res, PhxRequestTiming* timing) {
  return guarded([&]() -> int {
    if (!s) throw std::invalid_argument("null server");
    std::unique_ptr<Request> r;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      auto it = s->reqs.find(request);
      if (it == s->reqs.end()) throw std::invalid_argument("unknown request");
      if (it->second->state == PHX_REQ_FAILED) {
        const std::string e = it->second->error;
        s->reqs.erase(it);
        throw std::runtime_error(e);
      }
      if (it->second->state != PHX_REQ_DONE) throw std::invalid_argument("request not finished");
      r = std::move(it->second);
      s->reqs.erase(it);
    }
    if (res) std::memcpy(res, r->host.data(), r->host.size() * sizeof(PhxFreqOut));
    if (timing) *timing = r->t;
    return PHX_OK;
  });
}

int phx_server_stats(PhxServer* s, PhxServerStats* st) {
  return guarded([&]() -> int {
    if (!s || !st) throw std::invalid_argument("null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    *st = s->stats;
    st->inflight = s->inflight;
    st->pending = (int64_t)s->pending.size();
    st->generations = s->generations;
    st->arena_used = (int64_t)s->alloc->used();
    st->grid = s->lshape.grid;
    st->regs = s->lshape.regs;
    return PHX_OK;
  });
}

void phx_server_destroy(PhxServer* s) { delete s; }

}  // extern "C"
