// Camera: pixel -> impact parameters -> initial photon (FP64), and the polarization frames of an observer.
//
// The photon set-up is RAPTOR's distant-observer construction as the reference uses it (core/geometry/camera.hpp:
// 11-135): covariant Boyer-Lindquist wave vector from the impact parameters (alpha, beta) and the inclination,
// raised with the BL inverse metric at r_cam, k^r from the null condition, transformed to Kerr-Schild (log radius),
// and theta -> x2 inverted by Newton's method.  It runs once per ray, in FP64 in every precision mode.
#pragma once

#include "defs.cuh"
#include "kerr.cuh"

namespace phx {

// Impact parameters [r_g] of the centre of pixel (i, j) of a W x H image, then rotated by the position angle.
PHX_HD void pixel_impact(int i, int j, int W, int H, double fov_x, double fov_y, double cos_pa, double sin_pa,
                         double* alpha, double* beta) {
  const double a0 = -0.5 * fov_x + (i + 0.5) * fov_x / W;
  const double b0 = -0.5 * fov_y + (j + 0.5) * fov_y / H;
  *alpha = a0 * cos_pa + b0 * sin_pa;
  *beta = -a0 * sin_pa + b0 * cos_pa;
}

struct CameraSpec {
  double a, hslope;
  double incl_deg, phi_deg, r_cam, t_init;
};

PHX_HD double sign_of(double x) { return (x < 0.0) ? -1.0 : (x > 0.0) ? 1.0 : 0.0; }

// Newton inversion of theta = x2 + (h/2) sin 2 x2 (converged to 1e-15, at most 100 iterations).
PHX_HD double x2_of_theta(double hs, double th) {
  double cur = th, prev = 1e-15;
  for (int it = 0; it < 100 && fabs(cur - prev) > 1e-15; it++) {
    prev = cur;
    double s, c;
    sincos_t(2.0 * cur, &s, &c);
    cur = cur - (cur + 0.5 * hs * s - th) / (1.0 + hs * c);
  }
  return cur;
}

// k^theta -> k^{x2} (same Newton form as the position, which converges in one step since the map is linear).
PHX_HD double kx2_of_ktheta(double hs, double kth, double x2) {
  const double d = 1.0 + hs * cos_t(2.0 * x2);
  double cur = kth, prev = 1e-15;
  for (int it = 0; it < 100 && fabs(cur - prev) > 1e-15; it++) {
    prev = cur;
    cur = cur - (cur * d - kth) / d;
  }
  return cur;
}

// Photon (x^mu, k^mu) in MKS-BHAC at the camera for impact parameters (alpha, beta).
PHX_HD void camera_photon(const CameraSpec& cs, double alpha, double beta, double ph[8]) {
  const double a = cs.a, r = cs.r_cam;
  const double mu0 = cos_t(cs.incl_deg / 180.0 * kPi);
  const double th0 = acos_t(mu0);
  const double phi0 = cs.phi_deg / 180.0 * kPi;
  const double x1c = log_t(r);
  // covariant BL wave vector: k_t = -1, k_phi = l, k_theta from the Carter constant of the distant observer
  const double l = -alpha * sqrt_t(1.0 - mu0 * mu0);
  const double qc = beta * beta + mu0 * mu0 * (alpha * alpha - 1.0);
  const double st = sin_t(th0), ct = cos_t(th0);
  const double st2 = st * st, ct2 = ct * ct;
  const double kd0 = -1.0, kd3 = l;
  const double kd2 = sign_of(beta) * sqrt_t(fabs_t(qc - l * l * (ct2 / st2) + ct2));
  // BL inverse metric at (r, th0)
  const double sig = r * r + a * a * ct * ct;
  const double del = r * r + a * a - 2.0 * r;
  const double AA = (r * r + a * a) * (r * r + a * a) - del * a * a * st * st;
  const double g11 = sig / del * r * r;  // g_{x1 x1} of BL with log radius
  const double gtt = -AA / (sig * del);
  const double gtp = -2.0 * a * r / (sig * del);
  const double gpp = (del - a * a * st * st) / (sig * del * st * st);
  const double gthth = 1.0 / sig;
  const double ku0 = gtt * kd0 + gtp * kd3;
  const double ku3 = gpp * kd3 + gtp * kd0;
  const double ku2 = gthth * kd2;
  const double ku1 = sqrt_t((-ku0 * kd0 - ku2 * kd2 - ku3 * kd3) / g11);
  // BL -> KS (log radius)
  const double rp = exp_t(x1c);
  const double D = rp * rp - 2.0 * rp + a * a;
  const double sq = sqrt_t(1.0 - a * a);
  const double rplus = 1.0 + sq, rminus = 1.0 - sq;
  const double lg = log_t((rp - rplus) / (rp - rminus));
  ph[0] = cs.t_init + (log_t(D) + lg / sq);
  ph[1] = x1c;
  ph[2] = th0;
  ph[3] = phi0 + a / (2.0 * sq) * lg;
  ph[4] = ku0 + 2.0 * rp / D * rp * ku1;
  ph[5] = ku1;
  ph[6] = ku2;
  ph[7] = ku3 + a / D * rp * ku1;
  ph[2] = x2_of_theta(cs.hslope, ph[2]);
  ph[6] = kx2_of_ktheta(cs.hslope, ph[6], ph[2]);
}

// The two polarization axes seen by an observer with 4-velocity U looking along k, with reference direction b:
//   para = unit vector of b projected onto the screen,  perp = the screen vector orthogonal to it,
//   perp^mu = -eps^{mu nu rho sigma} U_nu k_rho b_sigma / (sqrt(-g) omega N)   (RAPTOR's observer tetrad, the
// reference's create_observer_tetrad, core/geometry/tetrad.hpp:51-101).  omega = -k.U is returned too.
template <class R>
PHX_HD void observer_axes_lowered(R sqrtg, const R k[4], const R U[4], const R b[4], const R kd[4], const R Ud[4],
                                  const R bd[4], R omega, R kb, R Ub, R bb, R perp[4], R para[4]) {
  const R iomega = fastm::rcp(omega);
  R eK[4];
  for (int i = 0; i < 4; i++) eK[i] = k[i] * iomega - U[i];
  const R Beta = Ub;
  const R Cc = kb * iomega - Beta;
  const R Nc = fastm::sqrt(bb + Beta * Beta - Cc * Cc);
  const R iNc = fastm::rcp(Nc);
  for (int i = 0; i < 4; i++) para[i] = (b[i] + Beta * U[i] - Cc * eK[i]) * iNc;
  const R s = -iomega * iNc * fastm::rcp(sqrtg);
  // generalized cross product: perp^i = (-1)^i det[U, k, b] over the three columns other than i
  const R m01 = kd[0] * bd[1] - kd[1] * bd[0], m02 = kd[0] * bd[2] - kd[2] * bd[0], m03 = kd[0] * bd[3] - kd[3] * bd[0];
  const R m12 = kd[1] * bd[2] - kd[2] * bd[1], m13 = kd[1] * bd[3] - kd[3] * bd[1], m23 = kd[2] * bd[3] - kd[3] * bd[2];
  perp[0] = s * (Ud[1] * m23 - Ud[2] * m13 + Ud[3] * m12);
  perp[1] = -s * (Ud[0] * m23 - Ud[2] * m03 + Ud[3] * m02);
  perp[2] = s * (Ud[0] * m13 - Ud[1] * m03 + Ud[3] * m01);
  perp[3] = -s * (Ud[0] * m12 - Ud[1] * m02 + Ud[2] * m01);
}

template <class R>
PHX_HD void observer_axes(const Cov<R>& g, R sqrtg, const R k[4], const R U[4], const R b[4], R perp[4], R para[4],
                          R* omega_out) {
  R Ud[4], kd[4], bd[4];
  symv(g, U, Ud);
  symv(g, k, kd);
  symv(g, b, bd);
  const R omega = -dot4(kd, U);
  observer_axes_lowered(sqrtg, k, U, b, kd, Ud, bd, omega, dot4(kd, b), dot4(Ud, b), dot4(bd, b), perp, para);
  *omega_out = omega;
}

// sqrt(-g) of MKS-BHAC: Sigma sin(theta) r theta'.
template <class R>
PHX_HD R sqrt_neg_g(const KerrPt<R>& p) {
  return p.sig * fabs_t(p.s) * p.r * p.tp;
}

// Camera polarization vector F1 (the 'perp' axis of the static-at-infinity camera observer with up = -e_phi),
// the reference's camera_basis (core/geometry/tetrad.hpp:111-133), evaluated in precision R.
template <class R>
PHX_HD void camera_pol(R a, R hs, const double ph[8], double F1[4]) {
  R X[4], k[4];
  for (int i = 0; i < 4; i++) {
    X[i] = R(ph[i]);
    k[i] = R(ph[4 + i]);
  }
  const KerrPt<R> p = kerr_point(a, hs, X[1], X[2]);
  const Cov<R> g = cov_metric(p, a);
  const Contra<R> u = contra_metric(p, a);
  // U_mu = (-1, 0, 0, sqrt(C)), C = -(1 + g^tt) / g^33 (g^{t phi} = 0 in these coordinates)
  const R C = -(R(1) + u.tt) / u.x33;
  const R Ud[4] = {R(-1), R(0), R(0), sqrt_t(C)};
  R U[4];
  raise(u, Ud, U);
  const R up[4] = {R(0), R(0), R(0), R(-1)};
  R perp[4], para[4], om;
  observer_axes(g, sqrt_neg_g(p), k, U, up, perp, para, &om);
  for (int i = 0; i < 4; i++) F1[i] = (double)perp[i];
}

}  // namespace phx
