/* FP64 CPU oracle for the PHOENIX raymarch path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference renderer's CPU path (nohgz/phoenix, src/core/ and src/host/io/bhac_io.hpp),
 * compiled as FP64 (ACCURACY=FP64).  It is the checker for the CUDA product: only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg may load it, and nothing in the product links it.  Each function names the reference
 * file:line it follows.  The restatement is pinned against the reference itself (the reference's own headers compiled
 * by oracle/build_ref.py into oracle/_ref/) and against committed golden vectors under tests/golden/.
 */
#ifndef PHX_ORACLE_H
#define PHX_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAX_FREQS 32
#define ORC_MAX_LEVELS 16

/* The run parameters the reference reads from config.toml (core/model/bhac.hpp:62-129, UserParams). */
typedef struct {
  double inclination, fov_x, fov_y, r_cam, t_init, pa, phi_cam;
  int32_t img_width, img_height;
  int32_t nfreqs;
  double frequencies[ORC_MAX_FREQS];
  double mass, distance;
  double stepsize;
  int32_t max_steps;
  double horizon_margin;
  int32_t max_order;
  double m_unit, r_low, r_high, beta_c, sigma_cut, thetae_min, thetae_max, rt_outer;
  int32_t nspin, bpol, nlevels, sfc;
} OrcParams;

/* One (pixel, frequency) result, binary-identical to the reference's FreqOut (core/render/pixel.hpp:26-29). */
typedef struct {
  double IQUV[4];
  double tau, tauF;
} OrcFreqOut;

typedef struct OrcModel OrcModel;

/* Reads a BHAC dump + grid file and decodes the primitives on the host (bhac_io.hpp:143-499). Returns NULL and
 * fills err (if not NULL, errlen bytes) on failure. */
OrcModel* orc_load(const char* dump, const char* grid, const OrcParams* params, char* err, int errlen);
void orc_free(OrcModel* m);

/* Renders the pixels idx[0..n) (idx = i * img_height + j) with `threads` OpenMP threads (<= 0: all).
 * out: n * nfreqs records in request order; stats: n * 3 int64 (steps, nplasma, bad); either may be NULL.
 * Returns the wall time in seconds of the pixel loop. */
double orc_render(const OrcModel* m, const int32_t* idx, int64_t n, OrcFreqOut* out, int64_t* stats, int threads);

/* Snapshot tables as the reference's Model holds them, for checking a product reader against the oracle's. */
int32_t orc_nleafs(const OrcModel* m);
int32_t orc_nlevels(const OrcModel* m);
void orc_level_dims(const OrcModel* m, int32_t level, int32_t dims[3]);
const int32_t* orc_level_map(const OrcModel* m, int32_t level);
const double* orc_lb(const OrcModel* m);
const double* orc_dxc(const OrcModel* m);
const double* orc_prim(const OrcModel* m); /* nleafs * cells * 8 */
void orc_scalars(const OrcModel* m, double out[16]); /* a, hslope, gam, cut_in, r_out, Ne, Bu, x_lo[1..3], x_hi[1..3], .. */
double orc_pixel_solid_angle(const OrcModel* m);

/* Pieces exposed for unit tests of the physics. */
void orc_bessel_ratios(double x, double* r10, double* r02);
void orc_metric_dd(double a, double hs, const double X[4], double g[4][4]);
void orc_metric_uu(double a, double hs, const double X[4], double g[4][4]);

#ifdef __cplusplus
}
#endif
#endif
