/* FP64 CPU oracle for the PHOENIX raymarch path -- TEST INFRASTRUCTURE ONLY (see phx_oracle.h).
 *
 * Restates, in C and in FP64, the reference renderer's per-pixel raymarch (nohgz/phoenix src/core/) and its BHAC
 * reader (src/host/io/bhac_io.hpp).  The arithmetic follows the reference expression by expression so that the
 * oracle reproduces the reference bit for bit on the same inputs (checked against oracle/_ref, the reference's own
 * headers compiled by oracle/build_ref.py).  One deliberate difference: the Bessel-function ratios K1/K2 and K0/K2
 * for 0.01 <= x < 30 come from the integral representation K_nu(x) = int_0^inf exp(-x cosh t) cosh(nu t) dt by the
 * trapezoid rule (double-precision accurate for these arguments) instead of the reference's tabulated Chebyshev fit
 * (core/numerics/bessel.hpp:118-148); the two agree to ~1e-15 relative.
 */
#define _GNU_SOURCE
#include "phx_oracle.h"

#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- constants (core/numerics/constants.hpp:22-81) */
static const double M_PROTON = 1.6726219e-24;
static const double M_ELECTRON = 9.1093829e-28;
static const double Q_ELECTRON = 4.80320425e-10;
static const double SPEED_OF_LIGHT = 2.99792458e10;
static const double H_PLANCK = 6.62606885e-27;
static const double G_GRAV = 6.674e-8;
static const double M_SUN = 1.989e33;
static const double KPC = 3.086e21;
#define H_OVER_MEC2 (H_PLANCK / (M_ELECTRON * SPEED_OF_LIGHT * SPEED_OF_LIGHT))
#define NU_CRIT_COEFF (3. * Q_ELECTRON / (4. * M_PI * M_ELECTRON * SPEED_OF_LIGHT))
#define JNU_COEFF (Q_ELECTRON * Q_ELECTRON / (2. * 1.73205080756887729353 * SPEED_OF_LIGHT))
#define PLASMA_FREQ2_COEFF (4. * M_PI * Q_ELECTRON * Q_ELECTRON / M_ELECTRON)
#define GYRO_FREQ_COEFF (Q_ELECTRON / (M_ELECTRON * SPEED_OF_LIGHT))

/* FP64 thresholds (core/numerics/precision.hpp:51-56) */
#define STEP_TINY 1e-160
#define STEP_BIG 1e100
#define TOL_SERIES 1e-18
#define TOL_ASYM 1e-17

/* --------------------------------------------------------------------------- model (core/model/bhac.hpp:131-173) */
struct OrcModel {
  OrcParams up;
  int nxlone[3];
  double xprobmin[3], xprobmax[3];
  double unit_L;
  int nleafs, ndim, nwini, nws, cells;
  int nx[3], ng[3];
  double *lb, *dxc, *prim;
  double a, hslope, gam, Ne, Bu, rhigh, rlow, ibc;
  int nlevels;
  int level_dims[ORC_MAX_LEVELS][3];
  int32_t* level_map[ORC_MAX_LEVELS];
  double lvl_w[ORC_MAX_LEVELS][3];
  double x_lo[4], x_hi[4];
  double cos_pa, sin_pa;
  double r_out, cut_in;
  double freq[ORC_MAX_FREQS], hconst[ORC_MAX_FREQS], jscale[ORC_MAX_FREQS];
};

static double sgn(double x) { return (x < 0.) ? -1. : (x > 0.) ? 1. : 0.; }

/* ---------------------------------------------------------------------------------- Bessel ratios (bessel.hpp) */
/* Scaled e^x K_{0,1,2}(x) by the trapezoid rule on the integral representation (the reference's small-x branch,
 * bessel.hpp:65-88). */
static void bessel_K012_scaled(double x, double* K0s, double* K1s, double* K2s) {
  const double dt = fmin(0.2, 0.7 / sqrt(x));
  const double tmax = acosh(1. + 42. / x) + 2.;
  const int nmax = (int)(tmax / dt) + 1;
  double s0 = 0.5, s1 = 0.5, s2 = 0.5;
  for (int k = 1; k <= nmax; k++) {
    const double t = (double)k * dt;
    const double sh2 = sinh(0.5 * t);
    const double ch = 1. + 2. * sh2 * sh2;
    const double e = exp(-2. * x * sh2 * sh2);
    s0 += e;
    s1 += e * ch;
    s2 += e * (2. * ch * ch - 1.);
    if (e * (2. * ch * ch) < TOL_SERIES * 0.1 * s2) break;
  }
  *K0s = dt * s0;
  *K1s = dt * s1;
  *K2s = dt * s2;
}

/* Hankel asymptotic series without its common prefactor (bessel.hpp:99-108). */
static double hankel_sum(int nu, double x) {
  const double mu = (double)(4 * nu * nu);
  double term = 1., sum = 1.;
  for (int k = 1; k <= 30; k++) {
    term *= (mu - (double)(2 * k - 1) * (double)(2 * k - 1)) / ((double)k * 8. * x);
    sum += term;
    if (fabs(term) < TOL_ASYM) break;
  }
  return sum;
}

/* K1/K2 and K0/K2 (bessel.hpp:118-148; the 0.01 <= x < 30 range by quadrature, see the file header). */
void orc_bessel_ratios(double x, double* r10, double* r02) {
  if (x >= 30.) {
    const double s2 = hankel_sum(2, x);
    *r10 = hankel_sum(1, x) / s2;
    *r02 = hankel_sum(0, x) / s2;
    return;
  }
  double k0, k1, k2;
  bessel_K012_scaled(x, &k0, &k1, &k2);
  *r10 = k1 / k2;
  *r02 = k0 / k2;
}

/* ---------------------------------------------------------------------------- metric (core/geometry/metric.hpp) */
/* metric_dd (metric.hpp:26-54) */
void orc_metric_dd(double a, double hs, const double X[4], double g[4][4]) {
  const double two = 2., one = 1.;
  const double r = exp(X[1]);
  const double s2x = sin(two * X[2]), c2x = cos(two * X[2]);
  const double th = X[2] + 0.5 * hs * s2x;
  const double s = sin(th), c = cos(th);
  const double s2 = s * s;
  const double rho2 = r * r + a * a * c * c;
  const double hfac = one + hs * c2x;
  memset(g, 0, 16 * sizeof(double));
  g[0][0] = -one + two * r / rho2;
  g[0][1] = g[1][0] = (two * r / rho2) * r;
  g[0][3] = g[3][0] = -two * a * r * s2 / rho2;
  g[1][1] = (one + two * r / rho2) * r * r;
  g[1][3] = g[3][1] = -a * s2 * (one + two * r / rho2) * r;
  g[2][2] = rho2 * hfac * hfac;
  g[3][3] = s2 * (rho2 + a * a * s2 * (one + two * r / rho2));
}

/* metric_uu (metric.hpp:64-92) */
void orc_metric_uu(double a, double hs, const double X[4], double g[4][4]) {
  const double two = 2., one = 1.;
  const double r = exp(X[1]);
  const double s2x = sin(two * X[2]), c2x = cos(two * X[2]);
  const double th = X[2] + 0.5 * hs * s2x;
  const double s = sin(th), c = cos(th);
  const double s2 = s * s;
  const double rho2 = r * r + a * a * c * c;
  const double hfac = one + hs * c2x;
  const double irho2 = one / rho2;
  memset(g, 0, 16 * sizeof(double));
  g[0][0] = -one - two * r * irho2;
  g[0][1] = g[1][0] = two * irho2;
  g[1][1] = irho2 * (r * (r - two) + a * a) / (r * r);
  g[1][3] = g[3][1] = a * irho2 / r;
  g[2][2] = irho2 / (hfac * hfac);
  g[3][3] = irho2 / s2;
}

/* metric_dd_uu (metric.hpp:103-143) */
static void metric_dd_uu(double a, double hs, const double X[4], double gd[4][4], double gu[4][4]) {
  const double two = 2., one = 1.;
  const double r = exp(X[1]);
  const double s2x = sin(two * X[2]), c2x = cos(two * X[2]);
  const double th = X[2] + 0.5 * hs * s2x;
  const double s = sin(th), c = cos(th);
  const double s2 = s * s;
  const double rho2 = r * r + a * a * c * c;
  const double irho2 = one / rho2;
  const double hfac = one + hs * c2x;
  memset(gd, 0, 16 * sizeof(double));
  memset(gu, 0, 16 * sizeof(double));
  gd[0][0] = -one + two * r / rho2;
  gd[0][1] = gd[1][0] = (two * r / rho2) * r;
  gd[0][3] = gd[3][0] = -two * a * r * s2 / rho2;
  gd[1][1] = (one + two * r / rho2) * r * r;
  gd[1][3] = gd[3][1] = -a * s2 * (one + two * r / rho2) * r;
  gd[2][2] = rho2 * hfac * hfac;
  gd[3][3] = s2 * (rho2 + a * a * s2 * (one + two * r / rho2));
  gu[0][0] = -one - two * r / rho2;
  gu[0][1] = gu[1][0] = two * irho2;
  gu[1][1] = irho2 * (r * (r - two) + a * a) / (r * r);
  gu[1][3] = gu[3][1] = a * irho2 / r;
  gu[2][2] = irho2 / (hfac * hfac);
  gu[3][3] = irho2 / s2;
}

/* inner_product, lower_index, raise_index, det4 (metric.hpp:148-213) */
static double inner_product(double g[4][4], const double* A, const double* B) {
  double s = 0.;
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) s += g[i][j] * A[i] * B[j];
  return s;
}
static void lower_index(double g[4][4], const double V[4], double out[4]) {
  for (int i = 0; i < 4; i++) {
    out[i] = 0.;
    for (int j = 0; j < 4; j++) out[i] += g[i][j] * V[j];
  }
}
static void raise_index(double g[4][4], const double V[4], double out[4]) { lower_index(g, V, out); }
static double det4(double m[4][4]) {
  const double s0 = m[2][0] * m[3][1] - m[2][1] * m[3][0];
  const double s1 = m[2][0] * m[3][2] - m[2][2] * m[3][0];
  const double s2 = m[2][0] * m[3][3] - m[2][3] * m[3][0];
  const double s3 = m[2][1] * m[3][2] - m[2][2] * m[3][1];
  const double s4 = m[2][1] * m[3][3] - m[2][3] * m[3][1];
  const double s5 = m[2][2] * m[3][3] - m[2][3] * m[3][2];
  const double c0 = m[0][0] * m[1][1] - m[0][1] * m[1][0];
  const double c1 = m[0][0] * m[1][2] - m[0][2] * m[1][0];
  const double c2 = m[0][0] * m[1][3] - m[0][3] * m[1][0];
  const double c3 = m[0][1] * m[1][2] - m[0][2] * m[1][1];
  const double c4 = m[0][1] * m[1][3] - m[0][3] * m[1][1];
  const double c5 = m[0][2] * m[1][3] - m[0][3] * m[1][2];
  return c0 * s5 - c1 * s4 + c2 * s3 + c3 * s2 - c4 * s1 + c5 * s0;
}

/* ------------------------------------------------------------------------------ camera (core/geometry/camera.hpp) */
static void pixel_impact(int i, int j, int w, int h, double fx, double fy, double* al, double* be) {
  *al = -0.5 * fx + (i + 0.5) * fx / w; /* camera.hpp:11-23 */
  *be = -0.5 * fy + (j + 0.5) * fy / h;
}

double orc_pixel_solid_angle(const OrcModel* m) { /* camera.hpp:28-32 */
  const double dist_cm = m->up.distance * KPC;
  return (m->up.fov_x / m->up.img_width * m->unit_L / dist_cm) * (m->up.fov_y / m->up.img_height * m->unit_L / dist_cm);
}

static double Xg2(double hs, double Xr2) { /* camera.hpp:37-46: Newton for x2(theta) */
  double cur = Xr2, prev = 1.e-15;
  int steps = 0;
  while (steps < 100 && fabs(cur - prev) > 1.e-15) {
    prev = cur;
    cur = cur - (cur + 0.5 * hs * sin(2. * cur) - Xr2) / (1. + hs * cos(2. * cur));
    steps++;
  }
  return cur;
}

static double Ug2(double hs, double Ur2, double Xg2v) { /* camera.hpp:51-61 */
  double cur = Ur2, prev = 1.e-15;
  int steps = 0;
  const double d = 1. + hs * cos(2. * Xg2v);
  while (steps < 100 && fabs(cur - prev) > 1.e-15) {
    prev = cur;
    cur = cur - (cur * d - Ur2) / d;
    steps++;
  }
  return cur;
}

static void initialize_photon(const OrcModel* m, double alpha, double beta, double ph[8]) { /* camera.hpp:71-135 */
  const double a = m->a;
  const double rcam = m->up.r_cam;
  const double mu0 = cos(m->up.inclination / 180. * M_PI);
  const double th0 = acos(mu0);
  const double phi0 = m->up.phi_cam / 180. * M_PI;
  const double Xc[4] = {m->up.t_init, log(rcam), th0, phi0};
  const double ll = -alpha * sqrt(1. - mu0 * mu0);
  const double qq = beta * beta + mu0 * mu0 * (alpha * alpha - 1.);
  const double sint = sin(th0), sinc2 = sint * sint, cost = cos(th0), cosc2 = cost * cost;
  const double kd0 = -1., kd3 = ll;
  const double kd2 = sgn(beta) * sqrt(fabs(qq - ll * ll * (cosc2 / sinc2) + cosc2));
  const double r = rcam, rfac = r;
  const double sigma = r * r + a * a * cost * cost;
  const double delta = r * r + a * a - 2. * r;
  const double A_ = (r * r + a * a) * (r * r + a * a) - delta * a * a * sint * sint;
  const double g11 = sigma / delta * rfac * rfac;
  const double guu00 = -A_ / (sigma * delta);
  const double guu03 = -2. * a * r / (sigma * delta);
  const double guu33 = (delta - a * a * sint * sint) / (sigma * delta * sint * sint);
  const double guu22 = 1. / sigma;
  const double ku0 = guu00 * kd0 + guu03 * kd3;
  const double ku3 = guu33 * kd3 + guu03 * kd0;
  const double ku2 = guu22 * kd2;
  const double ku1 = sqrt((-ku0 * kd0 - ku2 * kd2 - ku3 * kd3) / g11);
  const double rp = exp(Xc[1]);
  const double Del = rp * rp - 2. * rp + a * a;
  const double rplus = 1. + sqrt(1. - a * a);
  const double rmin = 1. - sqrt(1. - a * a);
  const double lg = log((rp - rplus) / (rp - rmin));
  ph[0] = Xc[0] + (log(Del) + lg / sqrt(1. - a * a));
  ph[1] = Xc[1];
  ph[2] = Xc[2];
  ph[3] = Xc[3] + a / (2. * sqrt(1. - a * a)) * lg;
  ph[4] = ku0 + 2. * rp / Del * rp * ku1;
  ph[5] = ku1;
  ph[6] = ku2;
  ph[7] = ku3 + a / Del * rp * ku1;
  ph[2] = Xg2(m->hslope, ph[2]);
  ph[6] = Ug2(m->hslope, ph[6], ph[2]);
}

/* ------------------------------------------------------------------------------ tetrad (core/geometry/tetrad.hpp) */
static void construct_U(const OrcModel* m, const double X[4], double U[4]) { /* tetrad.hpp:27-39 */
  double gu[4][4];
  orc_metric_uu(m->a, m->hslope, X, gu);
  const double Ud0 = -1.;
  const double B = -gu[0][3] * Ud0 / gu[3][3];
  const double C = -(1. + gu[0][0] * Ud0 * Ud0) / gu[3][3];
  const double Ud[4] = {Ud0, 0., 0., B + sqrt(B * B + C)};
  raise_index(gu, Ud, U);
}

static void create_observer_tetrad(const OrcModel* m, const double X[4], const double k[4], const double U[4],
                                   const double b[4], double e[4][4]) { /* tetrad.hpp:51-101 */
  double g[4][4];
  orc_metric_dd(m->a, m->hslope, X, g);
  const double omega = -inner_product(g, k, U);
  double eK[4];
  for (int i = 0; i < 4; i++) eK[i] = k[i] / omega - U[i];
  const double Beta = inner_product(g, U, b);
  const double Cc = inner_product(g, k, b) / omega - Beta;
  const double b2 = inner_product(g, b, b);
  const double Nc = sqrt(b2 + Beta * Beta - Cc * Cc);
  double para[4];
  for (int i = 0; i < 4; i++) para[i] = (b[i] + Beta * U[i] - Cc * eK[i]) / Nc;
  double Ud[4], kd[4], bd[4];
  lower_index(g, U, Ud);
  lower_index(g, k, kd);
  lower_index(g, b, bd);
  const double sq = sqrt(-det4(g));
  double perp[4];
  const double s = -1. / (sq * omega * Nc);
  static const int idx[4][3] = {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}};
  for (int i = 0; i < 4; i++) {
    const int a = idx[i][0], c = idx[i][1], d = idx[i][2];
    const double det = Ud[a] * (kd[c] * bd[d] - kd[d] * bd[c]) - Ud[c] * (kd[a] * bd[d] - kd[d] * bd[a]) +
                       Ud[d] * (kd[a] * bd[c] - kd[c] * bd[a]);
    perp[i] = ((i & 1) ? -s : s) * det;
  }
  for (int i = 0; i < 4; i++) {
    e[i][0] = U[i];
    e[i][1] = perp[i];
    e[i][2] = para[i];
    e[i][3] = eK[i];
  }
}

static void camera_basis(const OrcModel* m, const double X0[4], const double k0[4], double F1[4]) { /* tetrad.hpp:111-133 */
  double U[4], e[4][4];
  construct_U(m, X0, U);
  const double up[4] = {0., 0., 0., -1.};
  create_observer_tetrad(m, X0, k0, U, up, e);
  for (int i = 0; i < 4; i++) F1[i] = e[i][1];
}

static double pitch_angle(double g[4][4], const double k[4], const double B[4], const double U[4]) { /* tetrad.hpp:138-154 */
  const double Bn = sqrt(fabs(inner_product(g, B, B)));
  if (Bn == 0.) return M_PI / 2.;
  const double kk = fabs(inner_product(g, k, U));
  double mu = inner_product(g, k, B) / (kk * Bn);
  if (fabs(mu) > 1.) mu /= fabs(mu);
  return acos(mu);
}

static void chi_from_F1(double g[4][4], double e[4][4], const double F1[4], double* c2, double* s2) { /* tetrad.hpp:165-182 */
  double ep[4], ea[4];
  for (int mu = 0; mu < 4; mu++) {
    ep[mu] = e[mu][1];
    ea[mu] = e[mu][2];
  }
  const double C = inner_product(g, ep, F1);
  const double S = inner_product(g, ea, F1);
  const double n = C * C + S * S;
  *c2 = (C * C - S * S) / n;
  *s2 = 2. * C * S / n;
}

/* -------------------------------------------------------------------------- geodesic (core/geometry/geodesic.hpp) */
typedef struct {
  double a, a2, r, r2, tp, tp2, tpp, s, c, s2, s2th, cot, Sig, Sb, Delta, A, B, C;
} Geom;

static Geom make_geom(double a, double hslope, double x1, double x2) { /* geodesic.hpp:81-109 */
  Geom G;
  G.a = a;
  G.a2 = a * a;
  G.r = exp(x1);
  G.r2 = G.r * G.r;
  const double s2x = sin(2. * x2), c2x = cos(2. * x2);
  const double th = x2 + 0.5 * hslope * s2x;
  G.tp = 1. + hslope * c2x;
  G.tp2 = G.tp * G.tp;
  G.tpp = -2. * hslope * s2x;
  G.s = sin(th);
  G.c = cos(th);
  G.s2 = G.s * G.s;
  G.s2th = 2. * G.s * G.c;
  G.cot = G.c / G.s;
  G.Sig = G.r2 + G.a2 * G.c * G.c;
  G.Sb = 1. / G.Sig;
  G.Delta = G.r2 - 2. * G.r + G.a2;
  G.A = G.Sig * G.Delta + 2. * G.r * (G.r2 + G.a2);
  G.B = (2. * G.r2 - G.Sig) * G.Sb * G.Sb * G.Sb;
  G.C = G.r * G.Sb - G.a2 * G.B * G.s2;
  return G;
}

/* out[i] = -Gamma^i_jk U^j V^k, closed form in MKS-BHAC (geodesic.hpp:114-169) */
static void accel(const Geom* Gp, const double U[4], const double V[4], double out[4]) {
  const Geom G = *Gp;
  const double h = 0.5, two = 2., four = 4.;
  const double P00 = U[0] * V[0];
  const double P01 = h * (U[0] * V[1] + U[1] * V[0]);
  const double P02 = h * (U[0] * V[2] + U[2] * V[0]);
  const double P03 = h * (U[0] * V[3] + U[3] * V[0]);
  const double P11 = U[1] * V[1];
  const double P12 = h * (U[1] * V[2] + U[2] * V[1]);
  const double P13 = h * (U[1] * V[3] + U[3] * V[1]);
  const double P22 = U[2] * V[2];
  const double P23 = h * (U[2] * V[3] + U[3] * V[2]);
  const double P33 = U[3] * V[3];
  const double a = G.a, a2 = G.a2, r = G.r, r2 = G.r2, rp = G.r, rp2 = G.r2;
  const double tp = G.tp, tp2 = G.tp2, s = G.s, c = G.c, s2 = G.s2, s2th = G.s2th;
  const double Sig = G.Sig, Sb = G.Sb, Sb2 = Sb * Sb, Sb3 = Sb2 * Sb;
  const double Del = G.Delta, A = G.A, B = G.B, C = G.C, cot = G.cot;
  const double K = a2 * r * s2th * Sb2 * tp;
  out[0] = -two * (-r2 * Sb * tp2 * P22 - r * C * s2 * P33 + K * (-P02 - rp * P12 + a * s2 * P23) +
                   B * ((Sig + two * r) * rp * P01 + r * P00 + (Sig + r) * rp2 * P11 - two * a * r * s2 * P03 -
                        a * s2 * (Sig + two * r) * rp * P13));
  out[1] = -((1. - (two * Sig - Del) * B * rp) * P11 +
             (Del / rp) * (B * P00 - two * a * B * s2 * P03 - r * Sb * tp2 * P22 - C * s2 * P33) +
             two * ((Del - Sig) * B * P01 - a2 * s * c * Sb * tp * P12 + a * (r * Sb + (Sig - Del) * B) * s2 * P13));
  out[2] = -((G.tpp / tp - a2 * s * c * Sb * tp) * P22 +
             Sb3 *
                 ((-a2 * r * s2th) * (P00 + rp2 * P11) -
                  s * c * (Del * Sig * Sig + two * r * (r2 + a2) * (r2 + a2)) * P33 - two * a2 * r * s2th * rp * P01 +
                  two * a * s * c * (A + Sig * (Sig - Del)) * rp * P13 + two * a * r * (r2 + a2) * s2th * P03) /
                 tp +
             two * r * Sb * rp * P12);
  out[3] = -(a * (B * P00 + B * rp2 * P11 - r * Sb * tp2 * P22 - C * s2 * P33) + two * a * B * rp * P01 -
             four * a * r * cot * Sb2 * tp * P02 - two * a * (Sig + two * r) * cot * Sb2 * rp * tp * P12 -
             two * a2 * B * s2 * P03 + two * (cot + a2 * r * s2th * Sb2) * tp * P23 + two * C * rp * P13);
}

static void rhs(double a, double hs, const double y[8], const double f[4], double dy[8], double df[4]) {
  const Geom G = make_geom(a, hs, y[1], y[2]); /* geodesic.hpp:180-195 */
  const double* U = y + 4;
  double ag[4];
  for (int i = 0; i < 4; i++) dy[i] = U[i];
  accel(&G, U, U, ag);
  accel(&G, U, f, df);
  for (int i = 0; i < 4; i++) dy[4 + i] = ag[i];
}

/* One RK4 step of the FP64 state (x, k, F1) (geodesic.hpp:222-256; no hi/lo split and no pole folding at FP64). */
static void rk4_step(double a, double hs, double st[12], double dt) {
  double dy[4][8], dfr[4][4];
  double inc_y[8] = {0, 0, 0, 0, 0, 0, 0, 0}, inc_f[4] = {0, 0, 0, 0};
  const double w[3] = {0.5, 0.5, 1.0};
  for (int q = 0; q < 4; q++) {
    double ty[8], tf[4];
    for (int i = 0; i < 8; i++) ty[i] = st[i] + (0. + inc_y[i]);
    for (int i = 0; i < 4; i++) tf[i] = st[8 + i] + (0. + inc_f[i]);
    rhs(a, hs, ty, tf, dy[q], dfr[q]);
    if (q == 3) break;
    const double wdt = w[q] * dt;
    for (int i = 0; i < 8; i++) inc_y[i] = wdt * dy[q][i];
    for (int i = 0; i < 4; i++) inc_f[i] = wdt * dfr[q][i];
  }
  const double dt6 = dt / 6.;
  for (int i = 0; i < 8; i++) st[i] += ((dy[0][i] + dy[3][i]) + 2. * (dy[1][i] + dy[2][i])) * dt6;
  for (int i = 0; i < 4; i++) st[8 + i] += ((dfr[0][i] + dfr[3][i]) + 2. * (dfr[1][i] + dfr[2][i])) * dt6;
}

/* RAPTOR step-size rule with the AMR-cell cap (geodesic.hpp:267-292) */
static double step_size(double stepsize, const double X[4], const double k[4], const double* dxc) {
  const double S2 = STEP_TINY;
  const double dlx1 = stepsize / (fabs(k[1]) + S2);
  const double dlx2 = stepsize * fmin(X[2], M_PI - X[2]) / (fabs(k[2]) + S2);
  const double dlx3 = stepsize / (fabs(k[3]) + S2);
  const double i1 = 1. / (fabs(dlx1) + S2);
  const double i2 = 1. / (fabs(dlx2) + S2);
  const double i3 = 1. / (fabs(dlx3) + S2);
  double step_grid = STEP_BIG;
  if (dxc) {
    const double s1 = dxc[0] / (fabs(k[1]) + S2);
    const double s2 = dxc[1] / (fabs(k[2]) + S2);
    const double s3 = dxc[2] / (fabs(k[3]) + S2);
    const double is1 = 1. / (fabs(s1) + S2);
    const double is2 = 1. / (fabs(s2) + S2);
    const double is3 = 1. / (fabs(s3) + S2);
    step_grid = 1. / (is1 + is2 + is3) / 4.;
  }
  return -fmin(1. / (i1 + i2 + i3), step_grid);
}

static void normalize_null(double g[4][4], double k[4]) { /* geodesic.hpp:297-306 */
  const double aa = g[0][0];
  const double k1 = k[1], k2 = k[2], k3 = k[3];
  const double Betacap = -(g[0][1] * k1) / (aa) - (g[0][2] * k2) / (aa) - (g[0][3] * k3) / (aa);
  const double gz = -(g[1][1] * k1 * k1) / (aa) - (g[1][2] * k1 * k2) / (aa) - (g[1][3] * k1 * k3) / (aa) -
                    (g[2][1] * k2 * k1) / (aa) - (g[2][2] * k2 * k2) / (aa) - (g[2][3] * k2 * k3) / (aa) -
                    (g[3][1] * k3 * k1) / (aa) - (g[3][2] * k3 * k2) / (aa) - (g[3][3] * k3 * k3) / (aa);
  k[0] = Betacap + sqrt(Betacap * Betacap + gz);
}

/* ---------------------------------------------------------------------------- sampler (core/model/sampler.hpp) */
typedef struct {
  double U_u[4], B_u[4], n_e, B, theta_e, X_u[4];
} Fluid;

static void wrap_coords(double x[4]) { /* sampler.hpp:29-38 */
  const double TP = 2. * M_PI, PI = M_PI;
  x[3] = fmod(x[3], TP);
  x[2] = fmod(x[2], PI) - 1e-6;
  if (x[3] < 0.) x[3] = TP + x[3];
  if (x[2] < 0.) {
    x[2] = -x[2];
    x[3] = PI + x[3];
  }
}

static int outside_domain(const OrcModel* m, const double x[4]) { /* sampler.hpp:43-50 */
  return x[1] > m->x_hi[1] || x[1] < m->x_lo[1] || x[2] < m->x_lo[2] || x[2] > m->x_hi[2] || x[3] < m->x_lo[3] ||
         x[3] > m->x_hi[3];
}

static int find_leaf_map(const OrcModel* m, const double x[4]) { /* sampler.hpp:55-82 */
  double small = 1e-9;
  if (x[2] > M_PI / 2.) small = -small;
  const int top = m->nlevels - 1;
  const double up = (double)(1 << top);
  const double fi = (x[1] + small - m->x_lo[1]) / m->lvl_w[0][0] * up;
  const double fj = (x[2] + small - m->x_lo[2]) / m->lvl_w[0][1] * up;
  const double fk = (x[3] + small - m->x_lo[3]) / m->lvl_w[0][2] * up;
  if (fi < 0. || fj < 0. || fk < 0.) return -1;
  const int i = (int)fi, j = (int)fj, k = (int)fk;
  if (i >= m->level_dims[top][0] || j >= m->level_dims[top][1] || k >= m->level_dims[top][2]) return -1;
  for (int L = 0; L < m->nlevels; L++) {
    const int s = top - L;
    const int leaf =
        m->level_map[L][((size_t)(i >> s) * m->level_dims[L][1] + (j >> s)) * m->level_dims[L][2] + (k >> s)];
    if (leaf >= 0) return leaf;
  }
  return -1;
}

static int inside_leaf(const OrcModel* m, int leaf, const double x[4], double small) { /* sampler.hpp:87-101 */
  double lo[3], hi[3];
  for (int d = 0; d < 3; d++) {
    lo[d] = m->lb[3 * leaf + d];
    hi[d] = lo[d] + (double)m->nx[d] * m->dxc[3 * leaf + d];
  }
  return !(x[1] + small < lo[0] || x[1] + small >= hi[0] || x[2] + small < lo[1] || x[2] + small >= hi[1] ||
           x[3] + small < lo[2] || x[3] + small >= hi[2]);
}

static int inside_cached(const OrcModel* m, int leaf, const double x[4]) { /* sampler.hpp:109-122 */
  double lo[3], hi[3];
  for (int d = 0; d < 3; d++) {
    lo[d] = m->lb[3 * leaf + d];
    hi[d] = lo[d] + (double)m->nx[d] * m->dxc[3 * leaf + d];
  }
  return !(x[1] < lo[0] || x[1] > hi[0] || x[2] < lo[1] || x[2] > hi[1] || x[3] < lo[2] || x[3] > hi[2]);
}

static void find_cell3(const OrcModel* m, const double x[4], int leaf, int c[3]) { /* sampler.hpp:127-137 */
  for (int d = 0; d < 3; d++) {
    c[d] = (int)((x[1 + d] - m->lb[3 * leaf + d]) / m->dxc[3 * leaf + d]);
    if (c[d] >= m->nx[d]) c[d] = m->nx[d] - 1;
  }
}

static int find_leaf_scan(const OrcModel* m, const double x[4]) { /* sampler.hpp:143-157 */
  double small = 1e-9;
  if (x[2] > M_PI / 2.) small = -small;
  for (int leaf = 0; leaf < m->nleafs; leaf++)
    if (inside_leaf(m, leaf, x, small)) return leaf;
  return -1;
}

static int find_leaf(const OrcModel* m, const double x[4]) { /* sampler.hpp:162-180 */
  double small = 1e-9;
  if (x[2] > M_PI / 2.) small = -small;
  const int cand = find_leaf_map(m, x);
  if (cand >= 0 && inside_leaf(m, cand, x, small)) return cand;
  const double eps = 1e-6;
  if (cand < 0 && (x[1] < m->x_lo[1] - eps || x[1] > m->x_hi[1] + eps || x[2] < m->x_lo[2] - eps ||
                   x[2] > m->x_hi[2] + eps || x[3] < m->x_lo[3] - eps || x[3] > m->x_hi[3] + eps))
    return -1;
  return find_leaf_scan(m, x);
}

static int leaf_of(const OrcModel* m, const double X[4]) { /* sampler.hpp:182-192 */
  double x[4] = {X[0], X[1], X[2], X[3]};
  wrap_coords(x);
  if (exp(x[1]) < 1.) return -1;
  if (outside_domain(m, x)) return -1;
  return find_leaf(m, x);
}

static const double* grid_dxc(const OrcModel* m, const double X[4]) { /* sampler.hpp:198-206 */
  double x[4] = {X[0], X[1], X[2], X[3]};
  if (exp(x[1]) >= m->up.rt_outer) return NULL;
  wrap_coords(x);
  const int leaf = find_leaf(m, x);
  return leaf >= 0 ? &m->dxc[3 * leaf] : NULL;
}

static void sample_weights(const OrcModel* m, const double x[4], int leaf, double del[4]) { /* sampler.hpp:211-236 */
  double bs[3], dx[3];
  int ix[3];
  for (int d = 0; d < 3; d++) {
    bs[d] = m->lb[3 * leaf + d];
    dx[d] = m->dxc[3 * leaf + d];
  }
  for (int d = 0; d < 3; d++) {
    const double u = (x[1 + d] - bs[d]) / dx[d];
    ix[d] = (int)(u + 1000) - 1000;
  }
  for (int d = 0; d < 3; d++)
    del[1 + d] = (ix[d] < 0)                ? 0.
                 : (ix[d] > m->nx[d] - 2) ? 1.
                                          : (x[1 + d] - ((double)ix[d] * dx[d] + bs[d])) / dx[d];
}

static void interp_prims(const OrcModel* m, int leaf, const int c[3], const double del[4], double out[8]) {
  const int nx0 = m->nx[0], nx1 = m->nx[1], nx2 = m->nx[2]; /* sampler.hpp:260-291 */
  const int c_i = c[0], c_j = c[1], c_k = c[2];
  int c_ip = c_i + 1, c_jp = c_j + 1, c_kp = c_k + 1;
  if (c_ip >= nx0) c_ip = c_i;
  if (c_jp >= nx1) c_jp = c_j;
  if (c_kp >= nx2) c_kp = c_k;
  const double b1 = 1. - del[1], b2 = 1. - del[2], b3 = 1. - del[3];
  const int ci[4] = {c_i, c_i, c_ip, c_ip}, cj[4] = {c_j, c_jp, c_j, c_jp};
  const double wq[4] = {b1 * b2, b1 * del[2], del[1] * b2, del[1] * del[2]};
  const size_t lbase = (size_t)leaf * m->cells;
  for (int a = 0; a < 8; a++) out[a] = 0.;
  for (int z = 0; z < 2; z++) {
    const int ck = z ? c_kp : c_k;
    const double wz = z ? del[3] : b3;
    for (int q = 0; q < 4; q++) {
      const double* v = m->prim + (lbase + (ci[q] + cj[q] * nx0 + ck * nx0 * nx1)) * 8;
      const double w = wq[q] * wz;
      for (int a = 0; a < 8; a++) out[a] += v[a] * w;
    }
  }
}

static int derive_fluid(const OrcModel* m, const double x[4], double rho, double uu, const double Bp[4],
                        const double gV[4], Fluid* fl) { /* sampler.hpp:305-376 */
  const double smalll = 1.e-6;
  const double r = exp(x[1]);
  double gd[4][4], gu[4][4];
  metric_dd_uu(m->a, m->hslope, x, gd, gu);
  fl->n_e = rho * m->Ne + smalll;
  double shift[4];
  for (int j = 1; j < 4; j++) shift[j] = gu[0][j] / (-gu[0][0]);
  const double alpha = 1. / sqrt(-gu[0][0]);
  double gVdotgV = 0.;
  for (int i = 1; i < 4; i++)
    for (int j = 1; j < 4; j++) gVdotgV += gd[i][j] * gV[i] * gV[j];
  const double lfac = sqrt(gVdotgV + 1.);
  double V[4];
  for (int i = 1; i < 4; i++) V[i] = gV[i] / lfac;
  fl->U_u[0] = lfac / alpha;
  for (int i = 1; i < 4; i++) fl->U_u[i] = V[i] * lfac - shift[i] * lfac / alpha;
  fl->B_u[0] = 0.;
  for (int i = 1; i < 4; i++)
    for (int l = 1; l < 4; l++) fl->B_u[0] += lfac * Bp[i] * (gd[i][l] * V[l]) / alpha;
  for (int i = 1; i < 4; i++) fl->B_u[i] = (Bp[i] + alpha * fl->B_u[0] * fl->U_u[i]) / lfac;
  double Bd[4];
  lower_index(gd, fl->B_u, Bd);
  const double Bsq = fabs(fl->B_u[0] * Bd[0] + fl->B_u[1] * Bd[1] + fl->B_u[2] * Bd[2] + fl->B_u[3] * Bd[3]) + smalll;
  fl->B = sqrt(Bsq) * m->Bu;
  const double beta = uu * (m->gam - 1.) / (0.5 * (Bsq + smalll));
  const double bb = beta * m->ibc;
  const double b2 = bb * bb;
  const double trat = m->rhigh * b2 / (1. + b2) + m->rlow / (1. + b2);
  const double Thetae_unit = (1. / 3. * (M_PROTON / M_ELECTRON)) / (trat + 1.);
  fl->theta_e = (uu / rho) * Thetae_unit;
  if ((Bsq / (rho + 1e-20) > m->up.sigma_cut) || r > m->up.rt_outer || fl->theta_e > m->up.thetae_max ||
      fl->theta_e < m->up.thetae_min) {
    fl->n_e = 0.;
    return 0;
  }
  return 1;
}

static int get_fluid_params(const OrcModel* m, const double X[4], Fluid* fl, int* cache) { /* sampler.hpp:387-427 */
  double x[4] = {X[0], X[1], X[2], X[3]};
  wrap_coords(x);
  for (int i = 0; i < 4; i++) fl->X_u[i] = x[i];
  const double r = exp(x[1]);
  if (r < 1.) return 0;
  if (outside_domain(m, x)) return 0;
  int igrid = cache ? *cache : -1;
  if (igrid == -1 || !inside_cached(m, igrid, x)) {
    wrap_coords(x);
    igrid = find_leaf(m, x);
    if (cache) *cache = igrid;
  }
  for (int i = 0; i < 4; i++) fl->X_u[i] = x[i];
  if (igrid == -1) return 0;
  int c[3];
  find_cell3(m, x, igrid, c);
  double del[4], q[8];
  sample_weights(m, x, igrid, del);
  interp_prims(m, igrid, c, del, q);
  const double Bp[4] = {0., q[5], q[6], q[7]};
  const double gV[4] = {0., q[2], q[3], q[4]};
  return derive_fluid(m, x, q[0], q[1], Bp, gV, fl);
}

/* ---------------------------------------------------------------------------- transfer (core/transfer/coeffs.hpp) */
typedef struct {
  double jI, jQ, jU, jV, aI, aQ, aU, aV, rQ, rU, rV;
} PolCoeffs;

static const double COEF_C0 = 369.69342869090815; /* 2^(-1/3) / 3^(23/6) * 1e4 * pi (coeffs.hpp:41) */
static const double LOG120 = 4.787491742782046;   /* ln 120 (coeffs.hpp:42) */

static double I_I(double x) { /* coeffs.hpp:44-48 */
  const double cbrtx = cbrt(x), icbrtx = 1. / cbrtx;
  return 2.5651 * (1. + 1.92 * icbrtx + 0.9977 * icbrtx * icbrtx) * exp(-1.8899 * cbrtx);
}
static double I_Q(double x) { /* coeffs.hpp:50-54 */
  const double cbrtx = cbrt(x), icbrtx = 1. / cbrtx;
  return 2.5651 * (1. + 0.93193 * icbrtx + 0.499873 * icbrtx * icbrtx) * exp(-1.8899 * cbrtx);
}
static double I_V(double x) { /* coeffs.hpp:56-61 */
  const double cbrtx = cbrt(x), icbrtx = 1. / cbrtx;
  return (1.81348 * icbrtx * icbrtx * icbrtx + 3.42319 * icbrtx * icbrtx + 0.0292545 / sqrt(x) + 2.03773 * icbrtx) *
         exp(-1.8899 * cbrtx);
}
static double f_m(double X) { /* coeffs.hpp:63-70 */
  const double lx = log(X);
  const double ex = exp(-X / 47.2);
  return 2.011 * exp(-exp(1.035 * lx) / 4.7) - cos(X * 0.5) * exp(-exp(1.2 * lx) / 2.73) - 0.011 * ex +
         (0.011 * ex - COEF_C0 * exp(-8. / 3. * lx)) * 0.5 * (1. + tanh(10. * (lx - LOG120)));
}
static double planck_nu(double nu, double te) { /* coeffs.hpp:75-80 */
  const double pre = (2. * H_PLANCK) * nu * nu * nu / (SPEED_OF_LIGHT * SPEED_OF_LIGHT);
  const double xx = H_OVER_MEC2 * nu / te;
  return pre / (exp(xx) - 1.);
}

static PolCoeffs thermal_raw(double te, double ne, double nu, double B, double thB) { /* coeffs.hpp:95-138 */
  PolCoeffs r;
  memset(&r, 0, sizeof r);
  const double sth = sin(thB), cth = cos(thB);
  const double ite = 1. / te;
  const double nu_c = NU_CRIT_COEFF * B * sth * te * te;
  const double x = nu / nu_c;
  const double pref = JNU_COEFF * ne * nu * ite * ite;
  r.jI = pref * I_I(x);
  r.jQ = pref * I_Q(x);
  r.jV = (4. / 3.) * pref * ite * (cth / sth) * I_V(x);
  const double Bnu = planck_nu(nu, te);
  const double iB = 1. / Bnu;
  r.aI = r.jI * iB;
  r.aQ = r.jQ * iB;
  r.aV = r.jV * iB;
  const double iw = 1. / ((2 * M_PI) * nu);
  const double wp2 = PLASMA_FREQ2_COEFF * ne;
  const double omega0 = GYRO_FREQ_COEFF * B;
  const double Xe = te * sqrt(1.4142135623730951 * sth * ((1.e3 / (2. * M_PI)) * omega0 / nu));
  double kr1, kr0;
  if (ite < 1. / 5.) {
    const double k0 = -log(ite / 2.) - 0.5772, k1 = 1. / ite, k2 = 2. / ite / ite;
    kr1 = k1 / k2;
    kr0 = (k2 > 0.) ? k0 / k2 : 1.;
  } else {
    orc_bessel_ratios(ite, &kr1, &kr0);
  }
  const double q = omega0 * iw;
  const double wpw = wp2 * iw;
  r.rQ = (0.5 / SPEED_OF_LIGHT) * wpw * q * q * f_m(Xe) * (kr1 + 6. * te) * sth * sth;
  const double shgm = 1. - 0.11 * log(1. + 0.035 * Xe);
  r.rV = (1. / SPEED_OF_LIGHT) * wpw * q * (kr0 * shgm) * cth;
  return r;
}

static PolCoeffs invariant(PolCoeffs c, double nu_p, double jscale) { /* coeffs.hpp:147-164 */
  const double js = jscale / nu_p / nu_p;
  c.jI *= js;
  c.jQ *= js;
  c.jV *= js;
  c.aI *= nu_p;
  c.aQ *= nu_p;
  c.aV *= nu_p;
  c.rQ *= nu_p;
  c.rV *= nu_p;
  const double pf = sqrt(c.jQ * c.jQ + c.jV * c.jV) / c.jI;
  if (pf > 1.) {
    c.jQ /= (pf + 0.005);
    c.jU /= (pf + 0.005);
    c.jV /= (pf + 0.005);
  }
  return c;
}

static PolCoeffs rotate_to_camera(const PolCoeffs* c, double c2, double s2) { /* coeffs.hpp:173-182 */
  PolCoeffs r = *c;
  r.jQ = c2 * c->jQ + s2 * c->jU;
  r.jU = -s2 * c->jQ + c2 * c->jU;
  r.aQ = c2 * c->aQ + s2 * c->aU;
  r.aU = -s2 * c->aQ + c2 * c->aU;
  r.rQ = c2 * c->rQ + s2 * c->rU;
  r.rU = -s2 * c->rQ + c2 * c->rU;
  return r;
}

/* ------------------------------------------------------------------------ operators (core/transfer/operators.hpp) */
typedef struct {
  double A[4][4];
  double S[4];
} Acc;

static void mat4_vec(double A[4][4], const double v[4], double out[4]) {
  for (int i = 0; i < 4; i++) {
    out[i] = 0.;
    for (int j = 0; j < 4; j++) out[i] += A[i][j] * v[j];
  }
}
static void mat4_mul(double A[4][4], double B[4][4], double C[4][4]) {
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      double s = 0.;
      for (int k = 0; k < 4; k++) s += A[i][k] * B[k][j];
      C[i][j] = s;
    }
}
static void accumulate(Acc* acc, const Acc* seg) { /* operators.hpp:74-86 */
  double Tc[4], Tn[4][4];
  mat4_vec(acc->A, seg->S, Tc);
  for (int i = 0; i < 4; i++) acc->S[i] += Tc[i];
  mat4_mul(acc->A, (double(*)[4])seg->A, Tn);
  memcpy(acc->A, Tn, sizeof Tn);
}

static void inv4(double m[4][4], double out[4][4]) { /* Gauss-Jordan with partial pivoting (operators.hpp:118-153) */
  double A[4][8];
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      A[i][j] = m[i][j];
      A[i][4 + j] = (i == j) ? 1. : 0.;
    }
  for (int c = 0; c < 4; c++) {
    for (int r = c + 1; r < 4; r++)
      if (fabs(A[r][c]) > fabs(A[c][c]))
        for (int j = 0; j < 8; j++) {
          const double t = A[c][j];
          A[c][j] = A[r][j];
          A[r][j] = t;
        }
    const double d = A[c][c];
    for (int j = 0; j < 8; j++) A[c][j] /= d;
    for (int r = 0; r < 4; r++) {
      if (r == c) continue;
      const double f = A[r][c];
      for (int j = 0; j < 8; j++) A[r][j] -= f * A[c][j];
    }
  }
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) out[i][j] = A[i][4 + j];
}

static Acc trapezoid(double K[4][4], const double j[4], double h) { /* operators.hpp:158-176 */
  double P[4][4], N[4][4], Pinv[4][4], tmp[4];
  for (int i = 0; i < 4; i++)
    for (int k = 0; k < 4; k++) {
      const double id = (i == k) ? 1. : 0.;
      P[i][k] = id + 0.5 * h * K[i][k];
      N[i][k] = id - 0.5 * h * K[i][k];
    }
  inv4(P, Pinv);
  Acc r;
  mat4_mul(Pinv, N, r.A);
  mat4_vec(Pinv, j, tmp);
  for (int i = 0; i < 4; i++) r.S[i] = h * tmp[i];
  return r;
}

/* ---------------------------------------------------------------------------------- pixel (core/render/pixel.hpp) */
typedef struct {
  int i;
  double x[4], k[4], F1[4], dl;
} Sample;

typedef struct {
  Acc acc[ORC_MAX_FREQS];
  double tau_sum[ORC_MAX_FREQS], tauF_sum[ORC_MAX_FREQS];
  int nplasma, bad;
} PixelState;

static void process_sample(const OrcModel* m, PixelState* ps, const Sample* sm, int right_leaf) { /* pixel.hpp:52-123 */
  const int nf = m->up.nfreqs;
  double X[4], k[4], F1[4];
  for (int q = 0; q < 4; q++) {
    X[q] = sm->x[q];
    k[q] = sm->k[q];
    F1[q] = sm->F1[q];
  }
  const double r = exp(X[1]);
  double g[4][4];
  orc_metric_dd(m->a, m->hslope, X, g);
  if (fabs(inner_product(g, k, k)) > 1e-6 && r > 2.) normalize_null(g, k);

  Fluid fl;
  memset(&fl, 0, sizeof fl);
  int cache = right_leaf;
  const int in_volume = get_fluid_params(m, X, &fl, &cache);
  int emit = 0;
  double ratio = 0., c2 = 0., s2 = 0., pitch = 0.;
  if (in_volume && r < m->up.rt_outer) {
    double sg[4][4], e[4][4];
    orc_metric_dd(m->a, m->hslope, fl.X_u, sg);
    pitch = pitch_angle(sg, k, fl.B_u, fl.U_u);
    if (!(pitch == 0. || pitch == M_PI)) {
      create_observer_tetrad(m, fl.X_u, k, fl.U_u, fl.B_u, e);
      chi_from_F1(sg, e, F1, &c2, &s2);
      ratio = -inner_product(sg, k, fl.U_u);
      emit = 1;
    }
  }
  if (!emit) return;
  for (int f = 0; f < nf; f++) {
    const double nu_p = m->freq[f] * ratio;
    const PolCoeffs raw = thermal_raw(fl.theta_e, fl.n_e, nu_p, fl.B, pitch);
    const PolCoeffs inv = invariant(raw, nu_p, m->jscale[f]);
    const PolCoeffs seg = rotate_to_camera(&inv, c2, s2);
    const double h = sm->dl * m->hconst[f];
    double K[4][4] = {{seg.aI, seg.aQ, seg.aU, seg.aV},
                      {seg.aQ, seg.aI, seg.rV, -seg.rU},
                      {seg.aU, -seg.rV, seg.aI, seg.rQ},
                      {seg.aV, seg.rU, -seg.rQ, seg.aI}};
    const double jv[4] = {seg.jI, seg.jQ, seg.jU, seg.jV};
    const Acc op = trapezoid(K, jv, h);
    int finite = 1;
    for (int a = 0; a < 4; a++) {
      finite = finite && isfinite(op.S[a]);
      for (int b = 0; b < 4; b++) finite = finite && isfinite(op.A[a][b]);
    }
    if (!finite) {
      ps->bad++;
      continue;
    }
    accumulate(&ps->acc[f], &op);
    ps->tau_sum[f] += seg.aI * h;
    ps->tauF_sum[f] += fabs(seg.rV * h);
  }
  ps->nplasma++;
}

static void render_pixel(const OrcModel* m, double alpha, double beta, OrcFreqOut* out, int64_t st[3]) {
  const int nf = m->up.nfreqs; /* pixel.hpp:134-224 */
  for (int q = 0; q < nf; q++) memset(&out[q], 0, sizeof(OrcFreqOut));
  double ph[8], F1d[4];
  initialize_photon(m, alpha, beta, ph);
  camera_basis(m, ph, ph + 4, F1d);
  PixelState pst;
  PixelState* ps = &pst;
  for (int f = 0; f < nf; f++) {
    memset(&ps->acc[f], 0, sizeof(Acc));
    for (int i = 0; i < 4; i++) ps->acc[f].A[i][i] = 1.;
    ps->tau_sum[f] = ps->tauF_sum[f] = 0.;
  }
  double geo[12];
  for (int i = 0; i < 8; i++) geo[i] = ph[i];
  for (int i = 0; i < 4; i++) geo[8 + i] = F1d[i];
  ps->nplasma = ps->bad = 0;
  int steps = 0, turns = 0, terminate = 0;
  double thdot_prev = 0., dl_prev = 0.;
  const int beta_neg = beta < 0., beta_pos = beta > 0.;
  Sample pend;
  memset(&pend, 0, sizeof pend);
  pend.i = -1;
  for (;;) {
    Sample cur;
    for (int i = 0; i < 4; i++) {
      cur.x[i] = geo[i];
      cur.k[i] = geo[4 + i];
      cur.F1[i] = geo[8 + i];
    }
    cur.i = steps;
    cur.dl = dl_prev;
    const double r = exp(cur.x[1]);
    const int alive = r < m->r_out && r > m->cut_in && steps < m->up.max_steps && !terminate;
    if (pend.i >= 1) process_sample(m, ps, &pend, alive ? leaf_of(m, cur.x) : -1);
    pend = cur;
    if (!alive) break;
    if (thdot_prev * cur.k[2] < 0. && steps > 2) turns++;
    thdot_prev = cur.k[2];
    if ((beta_neg && turns > m->up.max_order) || (beta_pos && turns > (m->up.max_order + 1))) terminate = 1;
    const double* dxc = grid_dxc(m, cur.x);
    double X[4], k[4];
    for (int i = 0; i < 4; i++) {
      X[i] = cur.x[i];
      k[i] = cur.k[i];
    }
    X[2] = geo[2]; /* pole_x2 at FP64 (geodesic.hpp:200-205) */
    const double dl = step_size(m->up.stepsize, X, k, dxc);
    rk4_step(m->a, m->hslope, geo, dl);
    dl_prev = fabs(dl);
    steps++;
  }
  st[0] = steps;
  st[1] = ps->nplasma;
  st[2] = ps->bad;
  if (ps->nplasma > 0)
    for (int f = 0; f < nf; f++) {
      out[f].tau = ps->tau_sum[f];
      out[f].tauF = ps->tauF_sum[f];
      for (int q = 0; q < 4; q++) out[f].IQUV[q] = ps->acc[f].S[q];
    }
}

double orc_render(const OrcModel* m, const int32_t* idx, int64_t n, OrcFreqOut* out, int64_t* stats, int threads) {
  const int H = m->up.img_height, W = m->up.img_width, nf = m->up.nfreqs;
  const double t0 = omp_get_wtime();
  const int nt = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
  for (int64_t p = 0; p < n; p++) { /* host/render/jobs.hpp:57-89 */
    const int i = idx[p] / H, j = idx[p] % H;
    double a0, b0;
    pixel_impact(i, j, W, H, m->up.fov_x, m->up.fov_y, &a0, &b0);
    const double alpha = a0 * m->cos_pa + b0 * m->sin_pa;
    const double beta = -a0 * m->sin_pa + b0 * m->cos_pa;
    OrcFreqOut tmp[ORC_MAX_FREQS];
    int64_t st[3];
    render_pixel(m, alpha, beta, tmp, st);
    if (out) memcpy(out + p * nf, tmp, sizeof(OrcFreqOut) * nf);
    if (stats) memcpy(stats + 3 * p, st, sizeof st);
  }
  return omp_get_wtime() - t0;
}

/* ------------------------------------------------------------------------------- reader (host/io/bhac_io.hpp) */
static double get_detgamma(double a, double hs, double x, double y, double z) { /* bhac.hpp:178-192 */
  const double X[4] = {0., x, y, z};
  double g[4][4];
  orc_metric_dd(a, hs, X, g);
  const double det = g[1][1] * (g[2][2] * g[3][3] - g[3][2] * g[2][3]) - g[1][2] * (g[2][1] * g[3][3] - g[3][1] * g[2][3]) +
                     g[1][3] * (g[2][1] * g[3][2] - g[2][2] * g[3][1]);
  return sqrt(det);
}

static void coord_bar(const OrcModel* m, const double X[3], const double dxc[3], double Xb[3]) { /* bhac.hpp:202-235 */
  const double c1[3] = {1., 4., 1.}, s[3] = {-1., 0., 1.};
  double norm = 0., xb = 0., yb = 0., zb = 0.;
  for (int k = 0; k < 3; k++)
    for (int j = 0; j < 3; j++)
      for (int i = 0; i < 3; i++) {
        const double w = c1[i] * c1[j] * c1[k];
        const double x = X[0] + dxc[0] / 2. * s[i];
        const double y = X[1] + dxc[1] / 2. * s[j];
        const double z = X[2] + dxc[2] / 2. * s[k];
        const double dg = get_detgamma(m->a, m->hslope, x, y, z);
        norm += dg * w;
        xb += dg * w * x;
        yb += dg * w * y;
        zb += dg * w * z;
      }
  const double vol = (dxc[0] / 6.0) * (dxc[1] / 6.0) * (dxc[2] / 6.0);
  norm *= vol;
  Xb[0] = xb * (vol / norm);
  Xb[1] = yb * (vol / norm);
  Xb[2] = zb * (vol / norm);
}

static void convert2prim(const OrcModel* m, const double lb3[3], const double dxc3[3], const double* cons, int cell,
                         double* prim) { /* bhac.hpp:247-346 */
  const int cells = m->cells;
  const int LFAC = m->nwini - 2, XI = m->nwini - 1;
#define Cv(nw) (cons[(size_t)(nw) * cells + cell])
  const int loc[3] = {cell % m->nx[0], (cell / m->nx[0]) % m->nx[1], cell / (m->nx[0] * m->nx[1])};
  double X[3], dxc[3];
  for (int d = 0; d < 3; d++) {
    dxc[d] = dxc3[d];
    X[d] = lb3[d] + (loc[d] + 0.5) * dxc3[d];
  }
  for (int v = 0; v < 8; v++) prim[v] = 0.;
  if (exp(X[0]) > 1.0) {
    double Xb[3];
    coord_bar(m, X, dxc, Xb);
    const double Xu[4] = {0., Xb[0], Xb[1], Xb[2]};
    double gd[4][4], gu[4][4];
    metric_dd_uu(m->a, m->hslope, Xu, gd, gu);
    const double BS = Cv(1) * Cv(5) + Cv(2) * Cv(6) + Cv(3) * Cv(7);
    double Bsq = 0., Bd[4] = {0, 0, 0, 0}, Su[4] = {0, 0, 0, 0}, gam_uu[4][4];
    for (int i = 1; i < 4; i++)
      for (int j = 1; j < 4; j++) gam_uu[i][j] = gu[i][j] + gu[0][i] * gu[0][j] / (-gu[0][0]);
    for (int j = 1; j < 4; j++)
      for (int i = 1; i < 4; i++) {
        Su[j] += gam_uu[i][j] * Cv(1 + i - 1);
        Bd[j] += gd[i][j] * Cv(5 + i - 1);
      }
    for (int i = 1; i < 4; i++) Bsq += Bd[i] * Cv(5 + i - 1);
    const double gam = m->gam;
    const double lfac = Cv(LFAC), xi = Cv(XI);
    const double rho = Cv(0) / lfac;
    double uu = (gam - 1.) / gam * (xi / pow(lfac, 2.) - rho) / (gam - 1.);
    if (uu < 0) {
      uu = (Cv(8) / Cv(0)) * pow(rho, gam - 1) / (gam - 1.);
      if (uu < 0) uu = 1e-14;
    }
    const double den = xi + Bsq;
    prim[0] = rho;
    prim[1] = uu;
    prim[2] = (Su[1] / den + Cv(5) * BS / (xi * den)) * lfac;
    prim[3] = (Su[2] / den + Cv(6) * BS / (xi * den)) * lfac;
    prim[4] = (Su[3] / den + Cv(7) * BS / (xi * den)) * lfac;
    prim[5] = m->up.bpol * Cv(5);
    prim[6] = m->up.bpol * Cv(6);
    prim[7] = m->up.bpol * Cv(7);
  }
#undef Cv
}

static int load_grid(OrcModel* m, const char* path, char* err, int errlen) { /* bhac_io.hpp:143-174 */
  FILE* f = fopen(path, "r");
  if (!f) {
    snprintf(err, errlen, "cannot open grid file %s", path);
    return 0;
  }
  double v[10];
  int nv = 0;
  char line[4096];
  while (nv < 10 && fgets(line, sizeof line, f)) {
    char* last = NULL;
    for (char* tok = strtok(line, " \t\r\n"); tok; tok = strtok(NULL, " \t\r\n")) last = tok;
    if (last) v[nv++] = atof(last);
  }
  fclose(f);
  if (nv < 10) {
    snprintf(err, errlen, "%s: expected 10 lines", path);
    return 0;
  }
  for (int d = 0; d < 3; d++) {
    m->nxlone[d] = (int)v[d];
    m->xprobmin[d] = v[3 + d];
    m->xprobmax[d] = v[6 + d];
  }
  m->hslope = v[9];
  return 1;
}

typedef struct {
  int* ind;
  int* lev;
  int n, cap;
} LeafList;

static void push_leaf(LeafList* L, int lev, int i, int j, int k) {
  if (L->n == L->cap) {
    L->cap = L->cap ? 2 * L->cap : 1024;
    L->ind = (int*)realloc(L->ind, sizeof(int) * 3 * L->cap);
    L->lev = (int*)realloc(L->lev, sizeof(int) * L->cap);
  }
  L->ind[3 * L->n] = i;
  L->ind[3 * L->n + 1] = j;
  L->ind[3 * L->n + 2] = k;
  L->lev[L->n++] = lev;
}

static void read_node(FILE* f, int level, int i, int j, int k, LeafList* L, int* ok) { /* bhac_io.hpp:39-112 */
  if (!*ok) return;
  int is_leaf = 0;
  if (fread(&is_leaf, sizeof(int), 1, f) != 1) {
    *ok = 0;
    return;
  }
  if (is_leaf) {
    push_leaf(L, level, i, j, k);
    return;
  }
  for (int ich = 0; ich < 8; ich++)
    read_node(f, level + 1, 2 * i + ich % 2, 2 * j + ((int)(ich / 2.)) % 2, 2 * k + (int)(ich / 4.), L, ok);
}

static uint64_t morton3(unsigned a, unsigned b, unsigned c) { /* bhac_io.hpp:123-130 */
  uint64_t ans = 0;
  for (uint64_t i = 0; i < 21; ++i)
    ans |= (((uint64_t)a & ((uint64_t)1 << i)) << (2 * i)) | (((uint64_t)b & ((uint64_t)1 << i)) << (2 * i + 1)) |
           (((uint64_t)c & ((uint64_t)1 << i)) << (2 * i + 2));
  return ans;
}

typedef struct {
  uint64_t key;
  int n;
} MKey;
static int cmp_mkey(const void* x, const void* y) {
  const MKey *a = (const MKey*)x, *b = (const MKey*)y;
  return (a->key > b->key) - (a->key < b->key);
}

OrcModel* orc_load(const char* dump, const char* grid, const OrcParams* params, char* err, int errlen) {
  char dummy[256];
  if (!err) {
    err = dummy;
    errlen = sizeof dummy;
  }
  OrcModel* m = (OrcModel*)calloc(1, sizeof(OrcModel));
  m->up = *params;
  if (!load_grid(m, grid, err, errlen)) {
    free(m);
    return NULL;
  }
  FILE* f = fopen(dump, "rb");
  if (!f) {
    snprintf(err, errlen, "Can't open %s", dump);
    free(m);
    return NULL;
  }
  /* footer (bhac_io.hpp:350-381) */
  int idump, neq;
  double ddump;
  fseek(f, -40, SEEK_END);
  int ok = fread(&m->nleafs, 4, 1, f) == 1 && fread(&idump, 4, 1, f) == 1 && fread(&m->ndim, 4, 1, f) == 1 &&
           fread(&idump, 4, 1, f) == 1 && fread(&m->nwini, 4, 1, f) == 1 && fread(&m->nws, 4, 1, f) == 1 &&
           fread(&neq, 4, 1, f) == 1 && fread(&idump, 4, 1, f) == 1 && fread(&ddump, 8, 1, f) == 1;
  if (!ok || m->ndim != 3) {
    snprintf(err, errlen, "bad dump header");
    fclose(f);
    free(m);
    return NULL;
  }
  fseek(f, -40 - (m->ndim * 4 + neq * 8), SEEK_END);
  for (int d = 0; d < 3; d++) ok = ok && fread(&m->nx[d], 4, 1, f) == 1;
  double* neqpar = (double*)malloc(sizeof(double) * (neq > 0 ? neq : 1));
  for (int i = 0; i < neq; i++) ok = ok && fread(&neqpar[i], 8, 1, f) == 1;
  if (!ok || m->up.nspin < 0 || m->up.nspin >= neq) {
    snprintf(err, errlen, "short read in the dump header");
    fclose(f);
    free(neqpar);
    free(m);
    return NULL;
  }
  /* finalize_model (bhac_io.hpp:183-251) */
  const double spin = neqpar[m->up.nspin];
  m->a = spin;
  m->gam = neqpar[0];
  free(neqpar);
  for (int d = 1; d < 3; d++) {
    m->xprobmin[d] *= 2. * M_PI;
    m->xprobmax[d] *= 2. * M_PI;
  }
  m->cells = m->nx[0] * m->nx[1] * m->nx[2];
  for (int d = 0; d < 3; d++) {
    m->ng[d] = m->nxlone[d] / m->nx[d];
    m->x_lo[1 + d] = m->xprobmin[d];
    m->x_hi[1 + d] = m->xprobmax[d];
  }
  for (int l = 0; l < 16; l++)
    for (int d = 0; d < 3; d++) m->lvl_w[l][d] = (m->xprobmax[d] - m->xprobmin[d]) / m->ng[d] / (double)(1 << l);
  m->unit_L = G_GRAV * m->up.mass * M_SUN / SPEED_OF_LIGHT / SPEED_OF_LIGHT;
  const double rho_u = m->up.m_unit / pow(m->unit_L, 3);
  m->Bu = SPEED_OF_LIGHT * sqrt(4. * M_PI * rho_u);
  m->Ne = rho_u / (M_PROTON + M_ELECTRON);
  m->rhigh = m->up.r_high;
  m->rlow = m->up.r_low;
  m->ibc = 1. / m->up.beta_c;
  m->cos_pa = cos(m->up.pa / 180. * M_PI);
  m->sin_pa = sin(m->up.pa / 180. * M_PI);
  m->cut_in = (1. + sqrt(1. - spin * spin)) * (1. + m->up.horizon_margin);
  m->r_out = 1.1 * m->up.r_cam;
  const double c_const = m->unit_L * H_PLANCK / (M_ELECTRON * SPEED_OF_LIGHT * SPEED_OF_LIGHT);
  for (int q = 0; q < m->up.nfreqs; q++) {
    const double nu = m->up.frequencies[q];
    m->freq[q] = nu;
    m->hconst[q] = (M_ELECTRON * SPEED_OF_LIGHT * SPEED_OF_LIGHT) / (H_PLANCK * nu) * c_const;
    m->jscale[q] = nu * nu * nu;
  }
  /* forest walk (bhac_io.hpp:386-434) */
  const long size_blk = (long)m->cells * m->nwini * 8;
  const long stag = (long)(m->nx[0] + 1) * (m->nx[1] + 1) * (m->nx[2] + 1) * m->nws * 8;
  fseek(f, (long)m->nleafs * (size_blk + stag), SEEK_SET);
  LeafList L = {NULL, NULL, 0, 0};
  ok = 1;
  if (m->up.sfc) {
    const int nb = m->ng[0] * m->ng[1] * m->ng[2];
    MKey* keys = (MKey*)malloc(sizeof(MKey) * nb);
    int q = 0;
    for (int i = 0; i < m->ng[0]; i++)
      for (int j = 0; j < m->ng[1]; j++)
        for (int k = 0; k < m->ng[2]; k++) {
          keys[q].key = morton3(i, j, k);
          keys[q].n = (i * m->ng[1] + j) * m->ng[2] + k;
          q++;
        }
    qsort(keys, nb, sizeof(MKey), cmp_mkey);
    for (int b = 0; b < nb; b++) {
      const int n = keys[b].n;
      read_node(f, 1, n / (m->ng[1] * m->ng[2]), (n / m->ng[2]) % m->ng[1], n % m->ng[2], &L, &ok);
    }
    free(keys);
  } else {
    for (int k = 0; k < m->ng[2]; k++)
      for (int j = 0; j < m->ng[1]; j++)
        for (int i = 0; i < m->ng[0]; i++) read_node(f, 1, i, j, k, &L, &ok);
  }
  if (!ok || L.n != m->nleafs) {
    snprintf(err, errlen, "grid mismatch: tree has %d leaves, header says %d", L.n, m->nleafs);
    fclose(f);
    free(L.ind);
    free(L.lev);
    free(m);
    return NULL;
  }
  /* leaf geometry (bhac_io.hpp:436-453) */
  m->lb = (double*)malloc(sizeof(double) * 3 * m->nleafs);
  m->dxc = (double*)malloc(sizeof(double) * 3 * m->nleafs);
  double dx1[3], dxc0[3];
  for (int d = 0; d < 3; d++) {
    dx1[d] = (m->xprobmax[d] - m->xprobmin[d]) / m->ng[d];
    dxc0[d] = (m->xprobmax[d] - m->xprobmin[d]) / m->nxlone[d];
  }
  for (int l = 0; l < m->nleafs; l++) {
    const double inv_scale = 1.0 / (double)(1 << (L.lev[l] - 1));
    for (int d = 0; d < 3; d++) {
      m->lb[3 * l + d] = m->xprobmin[d] + L.ind[3 * l + d] * dx1[d] * inv_scale;
      m->dxc[3 * l + d] = dxc0[d] * inv_scale;
    }
  }
  /* level maps (bhac_io.hpp:257-309) */
  m->nlevels = m->up.nlevels;
  if (m->nlevels == -1)
    for (int l = 0; l < m->nleafs; l++)
      if (L.lev[l] > m->nlevels) m->nlevels = L.lev[l];
  if (m->nlevels < 1 || m->nlevels > 16) {
    snprintf(err, errlen, "%d AMR levels unsupported", m->nlevels);
    fclose(f);
    free(L.ind);
    free(L.lev);
    orc_free(m);
    return NULL;
  }
  m->up.nlevels = m->nlevels;
  for (int lvl = 0; lvl < m->nlevels; lvl++) {
    for (int d = 0; d < 3; d++) m->level_dims[lvl][d] = m->ng[d] * (1 << lvl);
    const size_t total = (size_t)m->level_dims[lvl][0] * m->level_dims[lvl][1] * m->level_dims[lvl][2];
    m->level_map[lvl] = (int32_t*)malloc(total * sizeof(int32_t));
    for (size_t t = 0; t < total; t++) m->level_map[lvl][t] = -1;
    for (int l = 0; l < m->nleafs; l++) {
      if (L.lev[l] - 1 != lvl) continue;
      const int i = L.ind[3 * l], j = L.ind[3 * l + 1], k = L.ind[3 * l + 2];
      if (i < 0 || i >= m->level_dims[lvl][0] || j < 0 || j >= m->level_dims[lvl][1] || k < 0 ||
          k >= m->level_dims[lvl][2])
        continue;
      m->level_map[lvl][(i * m->level_dims[lvl][1] + j) * m->level_dims[lvl][2] + k] = l;
    }
  }
  free(L.ind);
  free(L.lev);
  /* host decode (bhac_io.hpp:456-492) */
  m->prim = (double*)calloc((size_t)m->nleafs * m->cells * 8, sizeof(double));
  const size_t leaf_doubles = (size_t)m->nwini * m->cells;
  double* raw = (double*)malloc(sizeof(double) * leaf_doubles);
  fseek(f, 0, SEEK_SET);
  for (int l = 0; l < m->nleafs; l++) {
    if (fread(raw, sizeof(double), leaf_doubles, f) != leaf_doubles) {
      snprintf(err, errlen, "short read in the data, leaf %d", l);
      free(raw);
      fclose(f);
      orc_free(m);
      return NULL;
    }
    fseek(f, stag, SEEK_CUR);
#pragma omp parallel for schedule(static)
    for (int cell = 0; cell < m->cells; cell++)
      convert2prim(m, &m->lb[3 * l], &m->dxc[3 * l], raw, cell, &m->prim[((size_t)l * m->cells + cell) * 8]);
  }
  free(raw);
  fclose(f);
  return m;
}

void orc_free(OrcModel* m) {
  if (!m) return;
  free(m->lb);
  free(m->dxc);
  free(m->prim);
  for (int l = 0; l < ORC_MAX_LEVELS; l++) free(m->level_map[l]);
  free(m);
}

int32_t orc_nleafs(const OrcModel* m) { return m->nleafs; }
int32_t orc_nlevels(const OrcModel* m) { return m->nlevels; }
void orc_level_dims(const OrcModel* m, int32_t level, int32_t dims[3]) {
  for (int d = 0; d < 3; d++) dims[d] = m->level_dims[level][d];
}
const int32_t* orc_level_map(const OrcModel* m, int32_t level) { return m->level_map[level]; }
const double* orc_lb(const OrcModel* m) { return m->lb; }
const double* orc_dxc(const OrcModel* m) { return m->dxc; }
const double* orc_prim(const OrcModel* m) { return m->prim; }
void orc_scalars(const OrcModel* m, double out[16]) {
  out[0] = m->a;
  out[1] = m->hslope;
  out[2] = m->gam;
  out[3] = m->cut_in;
  out[4] = m->r_out;
  out[5] = m->Ne;
  out[6] = m->Bu;
  for (int d = 0; d < 3; d++) {
    out[7 + d] = m->x_lo[1 + d];
    out[10 + d] = m->x_hi[1 + d];
  }
  out[13] = m->unit_L;
  out[14] = m->nx[0];
  out[15] = m->cells;
}
