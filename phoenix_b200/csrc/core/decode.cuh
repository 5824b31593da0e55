// BHAC conserved -> primitive decode of one cell, FP64.
// Follows the reference's convert2prim (core/model/bhac.hpp:247-346): the metric is taken at the volume-weighted
// centroid of the cell (coord_bar, bhac.hpp:202-235: a 3x3x3 Simpson rule of sqrt(det gamma_ij)), the momentum is
// raised with the spatial inverse metric, and the stored Lorentz factor and xi = lfac^2 (rho + gamma u) give rho, u
// and u^i = lfac v^i.  The same routine runs on the host (dump reader) and on the device (decode kernel).
#pragma once

#include "defs.cuh"
#include "kerr.cuh"

namespace phx {

// Conserved slots of a BHAC dump (RAPTOR convention, bhac.hpp:26-36).  The last two slots of the nwini arrays are the
// auxiliary Lorentz factor and xi.
enum ConsSlot { kCD = 0, kCS1 = 1, kCS2 = 2, kCS3 = 3, kCTau = 4, kCB1 = 5, kCB2 = 6, kCB3 = 7, kCDS = 8 };

// sqrt(det gamma_ij): the x1-x3 block of the MKS metric has g_12 = g_23 = 0, so the determinant is
// g_22 (g_11 g_33 - g_13^2).
PHX_HD double sqrt_det_gamma(double a, double hs, double x1, double x2) {
  const KerrPt<double> p = kerr_point(a, hs, x1, x2);
  const Cov<double> g = cov_metric(p, a);
  return sqrt_t(g.x22 * (g.x11 * g.x33 - g.x13 * g.x13));
}

// Volume-weighted centroid of a cell with geometric centre X and size dx (Simpson weights 1-4-1 per axis).
PHX_HD void cell_centroid(double a, double hs, const double X[3], const double dx[3], double Xbar[3]) {
  const double w1[3] = {1.0, 4.0, 1.0};
  double norm = 0.0, s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (int k = 0; k < 3; k++) {
    const double z = X[2] + 0.5 * dx[2] * (k - 1);
    for (int j = 0; j < 3; j++) {
      const double y = X[1] + 0.5 * dx[1] * (j - 1);
      for (int i = 0; i < 3; i++) {
        const double x = X[0] + 0.5 * dx[0] * (i - 1);
        const double w = w1[i] * w1[j] * w1[k] * sqrt_det_gamma(a, hs, x, y);
        norm += w;
        s0 += w * x;
        s1 += w * y;
        s2 += w * z;
      }
    }
  }
  Xbar[0] = s0 / norm;
  Xbar[1] = s1 / norm;
  Xbar[2] = s2 / norm;
}

// Decode one cell.  cons points at the leaf's block (nwini arrays of `cells` doubles, cell = i + j nx0 + k nx0 nx1).
// lb3 / dx3: block origin and cell size of the leaf.  Writes kNPrim values (zero where r <= 1).
template <class P>
PHX_HD void cons_to_prim(double a, double hs, double gam, int bpol, int nwini, const int nx[3], const double lb3[3],
                         const double dx3[3], const double* cons, int cell, P* prim) {
  const int cells = nx[0] * nx[1] * nx[2];
  const int loc[3] = {cell % nx[0], (cell / nx[0]) % nx[1], cell / (nx[0] * nx[1])};
  double X[3];
  for (int d = 0; d < 3; d++) X[d] = lb3[d] + (loc[d] + 0.5) * dx3[d];
  for (int v = 0; v < kNPrim; v++) prim[v] = P(0);
  if (!(exp_t(X[0]) > 1.0)) return;

  double Xb[3];
  cell_centroid(a, hs, X, dx3, Xb);
  const KerrPt<double> p = kerr_point(a, hs, Xb[0], Xb[1]);
  const Cov<double> g = cov_metric(p, a);
  const Contra<double> u = contra_metric(p, a);

  auto C = [&](int slot) { return cons[(size_t)slot * cells + cell]; };
  const double S[4] = {0.0, C(kCS1), C(kCS2), C(kCS3)};
  const double B[4] = {0.0, C(kCB1), C(kCB2), C(kCB3)};
  // spatial inverse metric gamma^{ij} = g^{ij} - g^{0i} g^{0j} / g^{00} (g^{02} = g^{03} = 0 here)
  const double g11 = u.x11 - u.t1 * u.t1 / u.tt, g13 = u.x13, g22 = u.x22, g33 = u.x33;
  const double Su1 = g11 * S[1] + g13 * S[3];
  const double Su2 = g22 * S[2];
  const double Su3 = g13 * S[1] + g33 * S[3];
  // B_i = gamma_ij B^j, B^2 = B_i B^i
  double Bd[4];
  symv(g, B, Bd);
  const double Bsq = Bd[1] * B[1] + Bd[2] * B[2] + Bd[3] * B[3];
  const double BS = S[1] * B[1] + S[2] * B[2] + S[3] * B[3];

  const double lfac = C(nwini - 2), xi = C(nwini - 1);
  const double rho = C(kCD) / lfac;
  double uu = (xi / (lfac * lfac) - rho) / gam;
  if (uu < 0.0) {  // entropy fallback
    uu = (C(kCDS) / C(kCD)) * pow(rho, gam - 1.0) / (gam - 1.0);
    if (uu < 0.0) uu = 1e-14;
  }
  const double den = xi + Bsq;
  const double t = BS / (xi * den);
  prim[kRho] = P(rho);
  prim[kUU] = P(uu);
  prim[kU1] = P((Su1 / den + B[1] * t) * lfac);
  prim[kU2] = P((Su2 / den + B[2] * t) * lfac);
  prim[kU3] = P((Su3 / den + B[3] * t) * lfac);
  prim[kB1] = P(bpol * B[1]);
  prim[kB2] = P(bpol * B[2]);
  prim[kB3] = P(bpol * B[3]);
}

}  // namespace phx
