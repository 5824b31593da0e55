/* PHOENIX-B200: C ABI of the B200-native raymarch path of the PHOENIX GRRT renderer.
 *
 * The path: for each pixel, a null geodesic is marched from a distant camera towards a Kerr black hole with RK4 in
 * MKS-BHAC coordinates; at each step the block-AMR BHAC GRMHD snapshot is sampled and the polarized (I, Q, U, V)
 * thermal-synchrotron transfer operator is folded into the pixel's accumulator.  It replaces the reference's
 * device::render (nohgz/phoenix src/device/kernel.cuh:57-66, src/device/kernel.cu:284-360) and, for the CPU build,
 * host::jobs::process (src/host/render/jobs.hpp:50-92), both of which call core::pixel::render_pixel
 * (src/core/render/pixel.hpp:134-224) once per pixel.
 *
 * Conventions: every call returns 0 on success or a negative PHX_E* code, and phx_last_error() (per host thread)
 * describes the failure; nothing throws across this boundary.  Sizes are in elements unless stated.  Snapshots are
 * device-resident until destroyed.  One render at a time per snapshot handle and stream from one host thread.
 */
#ifndef PHOENIX_B200_H
#define PHOENIX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PHX_MAX_FREQS 32
#define PHX_MAX_LEVELS 16

enum {
  PHX_OK = 0,
  PHX_E_INVALID = -1,  /* bad argument (null pointer, size out of range, inconsistent tables) */
  PHX_E_IO = -2,       /* dump / grid file missing, short or malformed */
  PHX_E_CUDA = -3,     /* CUDA runtime error (no device, out of memory, launch failure) */
  PHX_E_TIMEOUT = -4,  /* a device wait ran out of iterations; the kernel returned early */
  PHX_E_UNSUPPORTED = -5
};

/* Arithmetic of a render. */
enum {
  PHX_PREC_FP32 = 0,  /* FP32 throughout after the FP64 camera set-up */
  PHX_PREC_FP64 = 1,  /* FP64 throughout */
  PHX_PREC_MIXED = 2  /* FP64 geodesic (state, RK4, step size, placement of samples in leaves and cells), FP32
                         plasma stage with FP64 null renormalisation, FP64 segment operators at large depth and
                         Kahan-summed Stokes vectors */
};

/* Snapshot creation flags. */
enum {
  PHX_SNAP_F64_PRIMS = 1, /* also keep FP64 primitives on the device (FP64 renders then read them) */
  PHX_SNAP_GPU_DECODE = 2 /* phx_snapshot_load: decode conserved -> primitive on the GPU while the dump streams in
                             (the reference's grmhd.gpu_decode, src/device/kernel.cu:105-112, 200-260) */
};

/* One (pixel, frequency) result; binary-identical to the reference's core::pixel::FreqOut
 * (src/core/render/pixel.hpp:26-29).  Stored at index (i * img_height + j) * nfreqs + f. */
typedef struct {
  double IQUV[4]; /* erg / s / cm^2 / Hz / sr (Jy / 1e23) */
  double tau, tauF;
} PhxFreqOut;

/* A decoded snapshot in host memory (what host::bhac_io::load leaves in the reference's core::bhac::Model,
 * src/core/model/bhac.hpp:131-173, src/host/io/bhac_io.hpp:331-499). */
typedef struct {
  int32_t nleafs;
  int32_t nx[3];       /* cells per block */
  int32_t ng[3];       /* base-level blocks per dimension */
  int32_t nlevels;     /* levels of the leaf maps */
  double a, hslope, gam;
  double x_lo[3], x_hi[3];           /* domain in (x1 = ln r, x2, x3), radians */
  const double* lb;                  /* [nleafs][3] block origins */
  const double* dxc;                 /* [nleafs][3] cell sizes */
  const float* prim_f32;             /* [nleafs][nx0*nx1*nx2][8] rho, u, u^1..3, B^1..3 (required) */
  const double* prim_f64;            /* same in FP64, or NULL */
  const int32_t* const* level_map;   /* nlevels maps, level L: [ng0<<L][ng1<<L][ng2<<L], leaf id or -1 */
} PhxSnapshotDesc;

/* Reader options (config.toml [grmhd] keys nspin, bpol, sfc, nlevels). */
typedef struct {
  int32_t nspin, bpol, sfc, nlevels;
} PhxReadOptions;

/* Everything a render reads besides the snapshot: the config.toml [camera], [black_hole], [integration] and
 * [plasma] keys (src/host/io/config.hpp:300-370), plus the precision and launch knobs of this library. */
typedef struct {
  /* [camera] */
  double inclination, fov_x, fov_y, r_cam, t_init, pa, phi;
  int32_t img_width, img_height;
  int32_t nfreqs;
  double frequencies[PHX_MAX_FREQS];
  /* [black_hole] */
  double mass, distance;
  /* [integration] */
  double stepsize;
  int32_t max_steps;
  double horizon_margin;
  int32_t max_order;
  /* [plasma] */
  double m_unit, r_low, r_high, beta_c, sigma_cut, thetae_min, thetae_max, rt_outer;
  /* this library */
  int32_t precision;   /* PHX_PREC_* */
  double r_fp64;       /* unused (kept for layout; the mixed mode integrates every step in FP64) */
  double tau_fp64;     /* mixed: FP64 segment operator where h max|K| exceeds this (<= 0: default 0.1) */
  int32_t block;       /* unused (the block shape follows blocks_per_sm; PhxRenderInfo.block reports it) */
  int32_t period;      /* march passes after which a warp refills its finished lanes even if others still run,
                          0 = default (2^20: longer than any ray, so a warp refills when it is empty) */
  int32_t blocks_per_sm; /* register-cap variant, as resident warps per SM / 4 (1: up to 255 registers in 128-thread
                            blocks; 3: 168 registers, 4: 128, as one 384 / 512-thread block per SM when the job list
                            fills every SM, else as 128-thread blocks); 0 = default (FP32 4; mixed 4 with one frequency, else 3;
                            FP64 1) */
  int32_t refill_lanes; /* a warp takes new jobs early, before the period ends, once this many of its 32 lanes have
                           finished (checked every 64 passes); 1..32, 0 = default (32: when the warp is empty) */
} PhxRenderParams;

/* What a render reports (a superset of the reference's device::Info, src/device/kernel.cuh:23-30). */
typedef struct {
  char device[256];
  int32_t sms, blocks, block, regs, local_bytes;
  double upload_s, kernel_s;
  int64_t steps, nplasma, bad;   /* sums over all rays */
  int64_t scans;                 /* leaf lookups that fell back to the linear scan */
  int64_t fp64_steps, fp64_ops;  /* mixed precision: RK4 steps and segment operators done in FP64 */
} PhxRenderInfo;

typedef struct PhxSnapshot PhxSnapshot;

/* Fills p with the reference's default config.toml values (input/config.toml) and PHX_PREC_FP32. */
void phx_default_params(PhxRenderParams* p);

/* Uploads a decoded snapshot and keeps it resident (replaces upload_model, src/device/kernel.cu:265-280). */
int phx_snapshot_create(const PhxSnapshotDesc* desc, int32_t flags, PhxSnapshot** out);

/* Reads a BHAC dump + grid file, decodes it on the host and uploads it (host::bhac_io::load_bhac_grid + load,
 * src/host/io/bhac_io.hpp:143-174, 331-499, then upload_model). */
int phx_snapshot_load(const char* dump_file, const char* grid_file, const PhxReadOptions* opt, int32_t flags,
                      PhxSnapshot** out);

void phx_snapshot_destroy(PhxSnapshot* s);

/* Host-only half of phx_snapshot_load: read and decode a BHAC dump into host memory (host::bhac_io::load with
 * gpu_decode = false, src/host/io/bhac_io.hpp:331-499).  phx_bhac_describe fills a descriptor whose pointers refer
 * into the host snapshot (valid until phx_bhac_free), ready for phx_snapshot_create on any device. */
typedef struct PhxHostSnapshot PhxHostSnapshot;
int phx_bhac_read(const char* dump_file, const char* grid_file, const PhxReadOptions* opt, int32_t flags,
                  PhxHostSnapshot** out);
int phx_bhac_describe(const PhxHostSnapshot* h, PhxSnapshotDesc* desc);
void phx_bhac_free(PhxHostSnapshot* h);

/* Device bytes held by a snapshot. */
int64_t phx_snapshot_bytes(const PhxSnapshot* s);

/* Shape, constants and load timings of a resident snapshot. */
typedef struct {
  int64_t nleafs;
  int32_t cells, nlevels, nx[3], ng[3];
  double a, hslope, gam, x_lo[3], x_hi[3];
  int32_t has_f64_prims, gpu_decoded;
  int64_t bytes;
  double read_s;    /* reading the dump (with the host decode when not decoded on the GPU) */
  double decode_s;  /* GPU decode: streaming the cells in, copies and decode kernels */
  double upload_s;  /* device allocation and uploads of phx_snapshot_create */
} PhxSnapshotInfo;
int phx_snapshot_info(const PhxSnapshot* s, PhxSnapshotInfo* info);

/* Copies the device primitives to host memory ([nleafs][cells][8]; either pointer may be NULL; prim_f64 needs a
 * snapshot with FP64 primitives). */
int phx_snapshot_download(const PhxSnapshot* s, float* prim_f32, double* prim_f64);

/* Pixel job list i * img_height + j, Morton-ordered (host::jobs::schedule with morton = true,
 * src/host/render/jobs.hpp:18-45).  jobs holds img_width * img_height entries. */
int phx_schedule_morton(int32_t img_width, int32_t img_height, int32_t* jobs);

/* Pixel job list in the order of a tile shape (PHX_TILE_*, below): PHX_TILE_MORTON is phx_schedule_morton; the others
 * cut the image into tiles of w x h pixels (w along i, h along j; j fastest inside a tile) and list the tiles in
 * Morton order of their coordinates, so that the 32 consecutive jobs a warp takes cover one tile.  No counterpart in
 * the reference, whose schedule is Morton only. */
int phx_schedule_tiles(int32_t img_width, int32_t img_height, int32_t tile_shape, int32_t* jobs);

/* Renders the pixels `jobs` (host array, NULL = every pixel in phx_default_pixel_order's order) into the host array res
 * (img_width * img_height * nfreqs records, index (i * img_height + j) * nfreqs + f; pixels not in jobs are left
 * untouched).  Synchronous.  Replaces device::render (src/device/kernel.cu:284-360). */
int phx_render(PhxSnapshot* s, const PhxRenderParams* p, const int32_t* jobs, int64_t njobs, PhxFreqOut* res,
               PhxRenderInfo* info);

/* Asynchronous form on a caller stream (cudaStream_t as void*, NULL = default stream) with device buffers:
 * d_jobs (njobs pixel indices), d_res (img_width * img_height * nfreqs records), d_pixstats (NULL or
 * 3 int32 per pixel: steps, nplasma, bad), d_counters (16 uint64, zeroed by the caller: queue head, steps, nplasma,
 * bad, scans, fp64_steps, fp64_ops, ...).  Allocates nothing. */
int phx_render_async(PhxSnapshot* s, const PhxRenderParams* p, const int32_t* d_jobs, int64_t njobs,
                     PhxFreqOut* d_res, int32_t* d_pixstats, uint64_t* d_counters, void* stream);

/* No counterpart in the reference, whose device::render allocates on every call.  For callers that cannot call
 * cudaMalloc -- a host application that owns all device memory through its own pool or arena, or a serving loop in
 * which an allocation would synchronize the device and stall other streams -- this entry point allocates nothing:
 * it stages `jobs` (host memory; pinned memory must stay valid until the stream has passed this call) and the
 * kernel's scratch (work-queue head, counters) in a fixed library-owned device array of 256 bytes plus
 * PHX_NOALLOC_MAX_JOBS job slots (4 MiB), which every GPU that loads the library holds until the process exits.
 * d_res: device buffer of img_width * img_height * nfreqs records.  Asynchronous on `stream` (NULL = default).
 * Rejects njobs > PHX_NOALLOC_MAX_JOBS with PHX_E_INVALID.  The first call on a device resolves the array's
 * device address with that device current.  The address is kept for the life of the process: do not call this entry point again on a device after cudaDeviceReset (the reset unloads
 * the library's module, and the kept address would be stale).  All calls share the
 * array (it keeps the last call's contents; the counter block is cleared before each launch), so calls that overlap
 * on the GPU race. */
#define PHX_NOALLOC_MAX_JOBS (1 << 20)
int phx_render_noalloc(PhxSnapshot* s, const PhxRenderParams* p, const int32_t* jobs, int64_t njobs,
                       PhxFreqOut* d_res, void* stream);

/* Per-frequency image totals of a device-resident result, computed on the device (the reference's
 * host::output::compute_spec and compute_tau, src/host/io/output.hpp:43-74): the flux line's I, Q, U, V [Jy] over
 * the pixels whose I+Q+U+V is finite, and the spectrum file's mean tau and tauF over the pixels whose six values are
 * finite.  Lets a caller that only wants the spectrum skip the image download (48 bytes per pixel and frequency). */
typedef struct {
  double IQUV[4];            /* total flux [Jy] */
  double tau_mean, tauF_mean;
  int64_t n_flux, n_tau;     /* pixels in the flux sums and in the optical-depth means */
} PhxSpectrum;

/* Reduces d_res (img_width * img_height * nfreqs records on the device, 16-byte aligned) into d_spec (nfreqs device
 * records), asynchronously on `stream` (NULL = default).  Allocates nothing; deterministic (fixed summation order). */
int phx_spectrum_async(const PhxRenderParams* p, const PhxFreqOut* d_res, PhxSpectrum* d_spec, void* stream);

/* ---- Batches: many images in one persistent, graph-captured launch ----
 * No single reference counterpart: the reference renders one image per device::render call
 * (src/device/kernel.cu:284-360, called once from src/main.cpp:186-187); a batch renders many such calls' images --
 * any mix of snapshots, resolutions, inclinations, frequencies and plasma parameters -- in one launch of a queue-fed
 * kernel whose lanes take rays from a device work queue of ray tiles, so that short images do not leave the GPU idle
 * while long rays finish.  Every item's result equals what phx_render returns for the same parameters, to the
 * rounding of the separately compiled kernel (and bit for bit across batches, whatever the mix). */
typedef struct PhxBatch PhxBatch;

typedef struct {
  PhxSnapshot* snapshot;   /* resident snapshot (all items on one device) */
  PhxRenderParams params;  /* one image; `precision` must agree across the batch; at most 4 frequencies unless FP32 */
  const int32_t* jobs;     /* host job list (copied at creation), or NULL: every pixel in Morton order */
  int64_t njobs;
} PhxBatchItem;

typedef struct {
  int32_t tile_rays;       /* rays per queue tile, 0 = 32 */
  int32_t blocks_per_sm;   /* register-cap variant (FP32: 1, 3, 4; mixed 1, 3, and 4 with one frequency slot),
                              0 = default (FP32 4; mixed 4 with one slot, else 3; FP64 1) or autotuned */
  int32_t period;          /* march passes after which a warp claims slots for its finished lanes even if others still
                              run, 0 = default (2^20) or autotuned */
  int32_t autotune;        /* nonzero: time every (blocks_per_sm, refill policy) candidate on a sample of the batch's
                              tiles at creation, then every tile shape at the fastest of them, and keep the fastest */
  int32_t sample_stride;   /* autotune sample: every n-th tile, 0 = 16 */
  int32_t keep_order;      /* nonzero: tiles in item order; 0: the largest images' tiles first */
  int32_t tile_shape;      /* pixel order of the items without a job list, i.e. the shape of the pixel tile a warp's
                              32 consecutive rays cover: PHX_TILE_* (0 = Morton, the reference's schedule) */
  int32_t lane_setup;      /* nonzero: each lane sets up the camera ray it takes (no start-state buffer); 0: a ray-setup
                              kernel sets up every job at full SIMD width before the queue kernel, in the same graph */
  int32_t refill_lanes;    /* a warp claims new slots early once this many of its lanes have finished (checked every 64
                              passes); 1..32, 0 = default (32: when the warp is empty) or autotuned */
} PhxBatchOptions;

/* Tile shapes: Morton (Z-order, 8x4-pixel warp tiles, the reference's host::jobs::schedule), or tiles of w x h pixels
 * (w along i, h along j; pixels j-fastest inside a tile), the tiles in Morton order of their coordinates.
 * PHX_TILE_CENTER_4X8: 4x8 tiles grouped in 32x32-pixel blocks, the blocks nearest the image centre first (ties in
 * Morton order), the tiles of a block in Morton order. */
enum {
  PHX_TILE_MORTON = 0,
  PHX_TILE_16X2 = 1,
  PHX_TILE_32X1 = 2,
  PHX_TILE_4X8 = 3,
  PHX_TILE_2X16 = 4,
  PHX_TILE_CENTER_4X8 = 5,
  PHX_TILE_SHAPES = 6
};
/* The pixel order (PHX_TILE_*) for an image, which phx_render uses when it is given no job list and the serving loop
 * uses for every request: PHX_TILE_CENTER_4X8 for images of up to 6 rays per lane of a full grid of the current
 * device (SMs x 512 lanes; 148 SMs if no device can be queried: 454,656 pixels on B200), Morton for larger ones and
 * for a NULL p.  A pixel's result does not depend on the order, but a launch ends when its last rays do: the longest
 * rays (photon ring, plunging orbits) sit near the image centre and the shortest at its edge, so centre-first blocks
 * start the long rays early and leave short ones for the end, which matters while an image is a few rays per lane.
 * On B200, FP32: 512^2 images 6-12 % faster than Morton at 10, 60 and 163 degrees; a 1024^2 image 5 % slower (the
 * jobs in flight then cover a thin ring instead of a compact patch of the image). */
int phx_default_pixel_order(const PhxRenderParams* p);

#define PHX_TUNE_MAX_CANDIDATES 16
typedef struct {
  int32_t blocks_per_sm, period, tile_rays;
  int32_t grid, block, regs, local_bytes;
  int32_t ncand;  /* candidates timed by the autotuner (0 if it did not run) */
  int32_t cand_blocks_per_sm[PHX_TUNE_MAX_CANDIDATES], cand_period[PHX_TUNE_MAX_CANDIDATES];
  double cand_ms[PHX_TUNE_MAX_CANDIDATES];
  int32_t tile_shape;  /* PHX_TILE_* in use */
  int32_t cand_tile_shape[PHX_TUNE_MAX_CANDIDATES];
  int64_t nitems, ntiles, nrays;
  int64_t device_bytes;  /* device memory the batch holds (tables, job lists, results) */
  int32_t refill_lanes;  /* refill threshold in use */
  int32_t cand_refill_lanes[PHX_TUNE_MAX_CANDIDATES];
} PhxBatchTuning;

void phx_default_batch_options(PhxBatchOptions* o);

/* Uploads the items' constants and job lists, allocates their device results, optionally autotunes, and captures the
 * launch (queue reset + kernel) in a CUDA graph. */
int phx_batch_create(const PhxBatchItem* items, int32_t nitems, const PhxBatchOptions* opt, PhxBatch** out);

/* Replays the captured launch on `stream` (cudaStream_t as void*, NULL = default stream).  Asynchronous. */
int phx_batch_launch(PhxBatch* b, void* stream);

/* Launch on the batch's own stream, wait, and record the kernel time (reported by phx_batch_result). */
int phx_batch_run(PhxBatch* b);

/* After a launch has completed: item `item`'s records into host memory res (img_width * img_height * nfreqs
 * records; pixels outside its job list are zero) and its counters into info (NULL allowed). */
int phx_batch_result(PhxBatch* b, int32_t item, PhxFreqOut* res, PhxRenderInfo* info);

/* Device address of item `item`'s records (valid until phx_batch_destroy). */
int phx_batch_device_result(PhxBatch* b, int32_t item, PhxFreqOut** d_res);

/* Item `item`'s per-frequency totals (nfreqs records in host memory), reduced on the device from the batch's last
 * run without downloading the image (see phx_spectrum_async).  Synchronous on the batch's stream. */
int phx_batch_spectrum(PhxBatch* b, int32_t item, PhxSpectrum* spec);

int phx_batch_tuning(const PhxBatch* b, PhxBatchTuning* t);

void phx_batch_destroy(PhxBatch* b);

/* ---- Serving: continuous batching of render requests ----
 * No reference counterpart (the reference renders one configured image per process run, src/main.cpp:120-205).  A
 * server keeps snapshots resident, admits requests first-in first-out by device memory (a result arena inside
 * memory_budget), and merges each admitted request's rays into one running queue kernel while earlier requests are
 * still on the GPU.  Each request's result equals what phx_render returns for it, to the rounding of the separately
 * compiled kernel, whatever else runs beside it.  The API is thread-safe; all CUDA work runs on the server's own
 * scheduler thread.  Large requests' tiles enter the queue a chunk at a time as it drains, and small requests enter
 * whole ahead of them, so a small request that arrives behind a large one does not wait for all of the large one. */
typedef struct PhxServer PhxServer;

enum { PHX_REQ_QUEUED = 0, PHX_REQ_RUNNING = 1, PHX_REQ_DONE = 2, PHX_REQ_FAILED = 3 };

typedef struct {
  int64_t memory_budget;  /* device bytes for snapshots, queue tables and the result arena (default 150 GiB) */
  int64_t arena_bytes;    /* results + job lists of requests in flight, 0 = min(what the budget leaves, 16 GiB) */
  int32_t precision;      /* PHX_PREC_*, shared by every request */
  int32_t max_freqs;      /* frequency slots per request (1 or 4; FP32 also up to 32), default 4 */
  int32_t tile_rays;      /* rays per queue tile, default 32 */
  int32_t period;         /* march passes after which a warp claims slots for its finished lanes, default 2^20 */
  int32_t blocks_per_sm;  /* register-cap variant, 0 = default (FP32 4; mixed 4 with one slot, else 3; FP64 1) */
  int32_t max_items;      /* requests per run of the kernel before the queue is recycled, default 4096 */
  int64_t max_tiles;      /* tiles per run of the kernel, a power of two, default 2^22 */
  int32_t idle_ns;        /* sleep of an idle warp between polls of the queue, default 2000 */
  int64_t idle_limit;     /* polls after which an idle warp stops waiting and the kernel leaves, default 5e6 */
  double linger_ms;       /* idle time after which the scheduler stops the kernel, default 20 */
  int32_t poll_us;        /* scheduler polling interval, default 50 */
  int32_t publish_chunk;  /* tiles a large request publishes at a time, default 64 */
  int64_t backlog_rays;   /* published but unclaimed rays kept in the queue, 0 = half a grid-load of lanes */
  int64_t small_rays;     /* requests of at most this many rays enter the queue whole, ahead of the large ones'
                             remaining tiles (default 65536, a 256^2 image) */
  int32_t refill_lanes;   /* a warp claims new slots early once this many of its lanes have finished, default 32 */
} PhxServerOptions;

typedef struct {
  double submitted_s;     /* submission time since the server was created */
  double admitted_s;      /* seconds from submission to publication into the queue */
  double done_s;          /* seconds from submission to the result being back in host memory */
  int64_t rays, steps, nplasma, bad;
} PhxRequestTiming;

typedef struct {
  int64_t submitted, completed, inflight, pending, generations;
  int64_t rays, steps;
  int64_t snapshot_bytes, table_bytes, arena_bytes, arena_used, job_table_bytes;
  int32_t grid, regs;
  int64_t idle_exits;  /* kernel runs that ended by their bounded idle wait (idle_limit polls) */
  int64_t retries;     /* requests put back in the queue because the kernel ended before finishing them */
} PhxServerStats;

void phx_default_server_options(PhxServerOptions* o);

/* Starts a server over nsnaps resident snapshots (not owned: keep them alive until phx_server_destroy). */
int phx_server_create(PhxSnapshot* const* snaps, int32_t nsnaps, const PhxServerOptions* opt, PhxServer** out);

/* Queues a render of snapshot `snapshot` (index into the creation list); returns at once with its id. */
int phx_server_submit(PhxServer* s, int32_t snapshot, const PhxRenderParams* p, int64_t* request);

/* Current state (PHX_REQ_*) of a request. */
int phx_server_poll(PhxServer* s, int64_t request, int32_t* state);

/* Waits until the request is done or failed, at most timeout_s seconds (<= 0: no limit); PHX_E_TIMEOUT if not done. */
int phx_server_wait(PhxServer* s, int64_t request, double timeout_s, int32_t* state);

/* A finished request's records (img_width * img_height * nfreqs, index (i * img_height + j) * nfreqs + f) and
 * timing; releases the request (its id is unknown afterwards). */
int phx_server_result(PhxServer* s, int64_t request, PhxFreqOut* res, PhxRequestTiming* timing);

int phx_server_stats(PhxServer* s, PhxServerStats* st);

/* Finishes the requests in flight, stops the kernel and frees the server's device memory. */
void phx_server_destroy(PhxServer* s);

/* Writes a render's outputs the way PHOENIX's write_output does (src/main.cpp:52-86, src/host/io/output.hpp):
 * `image` = "hdf5" -> outdir/img_data.h5 (RAPTOR block layout, block_size pixels per side; if it cannot be written the
 * text image is written instead), "text" -> outdir/image.dat (image_<f>.dat per frequency when nfreqs > 1),
 * "both", or "none"; always outdir/spectrum.dat.  flux (NULL or nfreqs x 4) receives the total I, Q, U, V [Jy]
 * per frequency.  The directory must exist. */
int phx_write_output(const PhxRenderParams* p, const PhxFreqOut* res, const char* outdir, const char* image,
                     int32_t block_size, double* flux);

/* No counterpart in the reference.  Measures the current GPU's FP32 issue rate [TFLOP/s] with independent FMA chains
 * on every SM (best of `repeats` timed launches after one warm-up): the measured denominator of the raymarch's FP32
 * roofline, taken on the box and at the clocks of the run that reports it. */
int phx_measure_fp32_peak(int32_t repeats, double* tflops);

/* Description of the last error on this host thread. */
const char* phx_last_error(void);

/* Library version string. */
const char* phx_version(void);

#ifdef __cplusplus
}
#endif
#endif
