// Render constants from the user parameters: units, horizon cut, per-frequency transfer scales
// (the reference's finalize_model, src/host/io/bhac_io.hpp:183-251) in the precision of the render.
#pragma once

#include <cmath>
#include <stdexcept>
#include <string>

#include "../../../include/phoenix_b200.h"
#include "../core/ray.cuh"

namespace phx {

struct Units {
  double L, rho, B, Ne;
};

inline Units units_of(const PhxRenderParams& p) {
  Units u;
  u.L = cgs::g_newton * p.mass * cgs::m_sun / cgs::c_light / cgs::c_light;
  u.rho = p.m_unit / std::pow(u.L, 3);
  u.B = cgs::c_light * std::sqrt(4.0 * kPi * u.rho);
  u.Ne = u.rho / (cgs::m_proton + cgs::m_electron);
  return u;
}

// Validates the parameters; throws std::invalid_argument with a message.
inline void check_params(const PhxRenderParams& p) {
  auto bad = [](const std::string& m) { throw std::invalid_argument(m); };
  if (p.img_width < 1 || p.img_height < 1) bad("image size must be positive");
  if ((long long)p.img_width * p.img_height > (1LL << 31) - 1) bad("image too large (more than 2^31 pixels)");
  if (p.nfreqs < 1 || p.nfreqs > PHX_MAX_FREQS) bad("nfreqs must be in 1..32");
  for (int f = 0; f < p.nfreqs; f++)
    if (!(p.frequencies[f] > 0.0) || !std::isfinite(p.frequencies[f])) bad("frequencies must be positive and finite");
  if (!(p.r_cam > 1.0)) bad("r_cam must exceed the horizon");
  if (p.max_steps < 0) bad("max_steps must be >= 0");
  if (!(p.stepsize > 0.0)) bad("stepsize must be > 0");
  if (!(p.beta_c > 0.0)) bad("beta_c must be > 0");
  if (!(p.mass > 0.0) || !(p.distance > 0.0) || !(p.m_unit > 0.0)) bad("mass, distance and m_unit must be > 0");
  if (p.precision < PHX_PREC_FP32 || p.precision > PHX_PREC_MIXED) bad("unknown precision mode");
  if (p.refill_lanes < 0 || p.refill_lanes > 32) bad("refill_lanes must be in 0..32");
}

// Integration limits and step-size constants of a geodesic in precision G (the reference's FP32 / FP64 thresholds,
// core/numerics/precision.hpp:51-56).
template <class G>
StepConsts<G> step_consts(const PhxRenderParams& p, double r_h) {
  StepConsts<G> c;
  c.stepsize = G(p.stepsize);
  c.inv_stepsize = G(1.0 / p.stepsize);
  c.cut_in = G(r_h * (1.0 + p.horizon_margin));
  c.r_out = G(1.1 * p.r_cam);
  c.rt_outer = G(p.rt_outer);
  c.tiny = sizeof(G) == 4 ? G(1e-30) : G(1e-160);
  c.big = sizeof(G) == 4 ? G(1e30) : G(1e100);
  return c;
}

template <class R>
RenderConsts<R> make_consts(const PhxRenderParams& p, double a, double hslope) {
  RenderConsts<R> rc;
  const Units u = units_of(p);
  rc.W = p.img_width;
  rc.H = p.img_height;
  rc.nfreqs = p.nfreqs;
  rc.max_steps = p.max_steps;
  rc.max_order = p.max_order;
  rc.fov_x = p.fov_x;
  rc.fov_y = p.fov_y;
  rc.cos_pa = std::cos(p.pa / 180.0 * kPi);
  rc.sin_pa = std::sin(p.pa / 180.0 * kPi);
  // the camera set-up sees the spin and hslope in the geodesic's precision (FP64 for FP64 and mixed renders)
  const bool geo64 = sizeof(R) == 8 || p.precision == PHX_PREC_MIXED;
  rc.cam.a = geo64 ? a : (double)R(a);
  rc.cam.hslope = geo64 ? hslope : (double)R(hslope);
  rc.cam.incl_deg = p.inclination;
  rc.cam.phi_deg = p.phi;
  rc.cam.r_cam = p.r_cam;
  rc.cam.t_init = p.t_init;
  const double r_h = 1.0 + std::sqrt(1.0 - a * a);
  rc.step = step_consts<R>(p, r_h);
  rc.step_d = step_consts<double>(p, r_h);
  rc.tau_fp64 = R(p.tau_fp64 > 0.0 ? p.tau_fp64 : 0.1);
  rc.pv.Ne = R(u.Ne);
  rc.pv.Bu = R(u.B);
  rc.pv.rhigh = R(p.r_high);
  rc.pv.rlow = R(p.r_low);
  rc.pv.ibc = R(1.0 / p.beta_c);
  rc.pv.sigma_cut = R(p.sigma_cut);
  rc.pv.thetae_min = R(p.thetae_min);
  rc.pv.thetae_max = R(p.thetae_max);
  rc.pv.rt_outer = R(p.rt_outer);
  const double c_const = u.L * cgs::h_planck / (cgs::m_electron * cgs::c_light * cgs::c_light);
  for (int f = 0; f < kMaxFreqs; f++) {
    const double nu = f < p.nfreqs ? p.frequencies[f] : 1.0;
    rc.freq[f] = R(nu);
    rc.hconst[f] = R((cgs::m_electron * cgs::c_light * cgs::c_light) / (cgs::h_planck * nu) * c_const);
    rc.jscale[f] = R(nu * nu * nu);
  }
  return rc;
}

// Solid angle of one pixel [sr] (core/geometry/camera.hpp:28-32).
inline double pixel_solid_angle(const PhxRenderParams& p) {
  const Units u = units_of(p);
  const double d = p.distance * cgs::kpc;
  return (p.fov_x / p.img_width * u.L / d) * (p.fov_y / p.img_height * u.L / d);
}

}  // namespace phx
