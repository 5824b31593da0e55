// Thermal synchrotron emission, absorption and Faraday coefficients of one plasma sample.
//
// Emissivities: the Dexter (2016, Appendix) fits of the thermal j_I, j_Q, j_V; absorption by Kirchhoff's law with
// the Planck function; Faraday rotation / conversion from the Shcherbakov (2008) fits with the modified-Bessel
// ratios K1/K2, K0/K2 at 1/Theta_e (asymptotic forms for Theta_e > 5).  The published fit constants are the ones the
// reference renderer uses (core/transfer/coeffs.hpp:41-138); the Bessel ratios come from this project's own
// Chebyshev table (bessel_table.inc, generated by tools/gen_bessel_table.py) and the Hankel series for x >= 30.
//
// Everything that does not depend on the observing frequency (angles, temperature factors, Bessel ratios, plasma
// and gyro frequencies) is computed once per sample; the per-frequency part is ~20 transcendentals.
#pragma once

#include "defs.cuh"

namespace phx {

template <class R>
struct BesselPiece {
  R a, b, la, lb;
  int n64, n32;
  R c10[23], c02[23];
};

}  // namespace phx

#include "bessel_table.inc"

namespace phx {

#if defined(__CUDACC__)
__device__ const BesselPiece<float> kBesselF[PHX_BESSEL_NPIECE] = PHX_BESSEL_DATA;
__device__ const BesselPiece<double> kBesselD[PHX_BESSEL_NPIECE] = PHX_BESSEL_DATA;
#endif
static const BesselPiece<float> kBesselF_host[PHX_BESSEL_NPIECE] = PHX_BESSEL_DATA;
static const BesselPiece<double> kBesselD_host[PHX_BESSEL_NPIECE] = PHX_BESSEL_DATA;

template <class R>
PHX_HD const BesselPiece<R>* bessel_table() {
#if defined(__CUDA_ARCH__)
  if constexpr (sizeof(R) == 4) return kBesselF; else return kBesselD;
#else
  if constexpr (sizeof(R) == 4) return kBesselF_host; else return kBesselD_host;
#endif
}

// Hankel asymptotic series of K_nu(x) without its common factor sqrt(pi / 2x) e^-x (Abramowitz & Stegun 9.7.2).
template <class R>
PHX_HD R hankel_sum(int nu, R x, R tol) {
  const R mu = R(4 * nu * nu);
  R term = R(1), sum = R(1);
  for (int k = 1; k <= 30; k++) {
    term *= (mu - R(2 * k - 1) * R(2 * k - 1)) / (R(k) * R(8) * x);
    sum += term;
    if (fabs_t(term) < tol) break;
  }
  return sum;
}

template <class R>
struct RatioPair {
  R r10, r02;
};

// K1/K2 and K0/K2 from the Hankel series (x >= 30: Theta_e < 1/30), out of line: cool plasma is a minority of the
// samples and its series loops would otherwise sit in the march loop's instruction stream.
template <class R>
PHX_HD_OUTLINE RatioPair<R> bessel_ratios_hankel(R x) {
  const R tol = sizeof(R) == 4 ? R(1e-8) : R(1e-17);
  const R s2 = hankel_sum(2, x, tol);
  return {hankel_sum(1, x, tol) / s2, hankel_sum(0, x, tol) / s2};
}

// K1(x)/K2(x) and K0(x)/K2(x) for x >= 0.2 (x = 1/Theta_e; hotter plasma never calls this).
template <class R>
PHX_HD void bessel_ratios(R x, R* r10, R* r02) {
  if (x >= R(30)) {
    const RatioPair<R> rp = bessel_ratios_hankel(x);
    *r10 = rp.r10;
    *r02 = rp.r02;
    return;
  }
  const BesselPiece<R>* T = bessel_table<R>();
  int p = 0;
#pragma unroll
  for (int q = 1; q < PHX_BESSEL_NPIECE; q++)
    if (x >= T[q].a) p = q;
  const BesselPiece<R>* pc = T + p;
  const R la = pc->la, lb = pc->lb;
  const R z = fastm::div(R(2) * log_t(x) - (lb + la), lb - la);
  const int n = sizeof(R) == 4 ? pc->n32 : pc->n64;
  R b1a = R(0), b2a = R(0), b1b = R(0), b2b = R(0);
  for (int j = n - 1; j >= 1; j--) {
    const R ta = R(2) * z * b1a - b2a + pc->c10[j];
    b2a = b1a;
    b1a = ta;
    const R tb = R(2) * z * b1b - b2b + pc->c02[j];
    b2b = b1b;
    b1b = tb;
  }
  *r10 = pc->c10[0] + z * b1a - b2a;
  *r02 = pc->c02[0] + z * b1b - b2b;
}

// Frequency-independent part of the coefficients of one sample.
template <class R>
struct SynchroSample {
  R sth, cth;      // sin, cos of the pitch angle
  R ite;           // 1 / Theta_e
  R te;            // Theta_e
  R inu_c;         // 1 / nu_c, nu_c = 3 e B sin(theta) Theta_e^2 / (4 pi m_e c)
  R jpre;          // e^2 / (2 sqrt3 c) n_e / Theta_e^2   (j = jpre nu I(x))
  R kr1, kr0;      // K1/K2, K0/K2
  R wp2;           // plasma frequency^2
  R omega0;        // gyro frequency
};

// sth, cth: sine and cosine of the pitch angle (computed from its cosine directly; no angle is formed).
template <class R>
PHX_HD SynchroSample<R> synchro_sample(R te, R ne, R B, R sth, R cth) {
  constexpr double NU_CRIT = 3.0 * cgs::q_electron / (4.0 * kPi * cgs::m_electron * cgs::c_light);
  constexpr double JNU = cgs::q_electron * cgs::q_electron / (2.0 * 1.73205080756887729353 * cgs::c_light);
  constexpr double WP2 = 4.0 * kPi * cgs::q_electron * cgs::q_electron / cgs::m_electron;
  constexpr double GYRO = cgs::q_electron / (cgs::m_electron * cgs::c_light);
  SynchroSample<R> s;
  s.sth = sth;
  s.cth = cth;
  s.te = te;
  s.ite = fastm::rcp(te);
  s.inu_c = fastm::div(R(1), R(NU_CRIT) * B * s.sth * te * te);
  s.jpre = R(JNU) * ne * s.ite * s.ite;
  if (s.ite < R(1.0 / 5.0)) {
    // Theta_e > 5: K_nu(x) -> 2^(nu-1) (nu-1)! x^-nu (nu > 0), K_0 -> -ln(x/2) - gamma_E
    const R k0 = -log_t(s.ite * R(0.5)) - R(0.5772), k1 = fastm::rcp(s.ite), k2 = R(2) * k1 * k1;
    s.kr1 = fastm::div(k1, k2);
    s.kr0 = (k2 > R(0)) ? fastm::div(k0, k2) : R(1);
  } else {
    bessel_ratios(s.ite, &s.kr1, &s.kr0);
  }
  s.wp2 = R(WP2) * ne;
  s.omega0 = R(GYRO) * B;
  return s;
}

// Plasma-frame coefficients at frequency nu (cgs), already in the Lorentz-invariant form (j / nu^2 * nu^3 scaling
// folded in by jscale, alpha and rho times nu) and with the polarized emissivity clamped to |j_pol| <= j_I.
template <class R>
struct Coeffs {
  R jI, jQ, jV, aI, aQ, aV, rQ, rV;
};

template <class R>
PHX_HD Coeffs<R> synchro_coeffs(const SynchroSample<R>& s, R nu, R jscale) {
  constexpr double H_OVER_MEC2 = cgs::h_planck / (cgs::m_electron * cgs::c_light * cgs::c_light);
  constexpr double C0 = 369.69342869090815;  // 2^(-1/3) 3^(-23/6) 1e4 pi (Dexter 2016 f_m fit)
  constexpr double LOG120 = 4.787491742782046;
  Coeffs<R> c;
  // emissivity fits in x = nu / nu_c
  const R x = nu * s.inu_c;
  // cbrt stays accurate: exp(-1.8899 cbrt(x)) multiplies its relative error by 1.89 cbrt(x) ~ 10..100
  const R cx = cbrt_t(x), icx = fastm::div(R(1), cx);
  const R ex = fastm::exp(R(-1.8899) * cx);
  const R pref = s.jpre * nu;
  const R II = R(2.5651) * (R(1) + R(1.92) * icx + R(0.9977) * icx * icx) * ex;
  const R IQ = R(2.5651) * (R(1) + R(0.93193) * icx + R(0.499873) * icx * icx) * ex;
  const R IV = (R(1.81348) * icx * icx * icx + R(3.42319) * icx * icx + R(0.0292545) * fastm::rsqrt(x) +
                R(2.03773) * icx) * ex;
  R jI = pref * II;
  R jQ = pref * IQ;
  R jV = R(4.0 / 3.0) * pref * s.ite * fastm::div(s.cth, s.sth) * IV;
  // Kirchhoff: alpha = j / B_nu(Theta_e)
  // (2 h nu^3) / c^2 in this order: 2 h / c^2 alone (1.5e-47) is below the FP32 range
  const R pre = R(2.0 * cgs::h_planck) * nu * nu * nu * R(1.0 / (cgs::c_light * cgs::c_light));
  const R xx = R(H_OVER_MEC2) * nu * s.ite;
  const R iB = fastm::div(sizeof(R) == 4 ? expm1_t(xx) : (exp_t(xx) - R(1)), pre);
  R aI = jI * iB, aQ = jQ * iB, aV = jV * iB;
  // Faraday rotation / conversion
  const R iw = fastm::div(R(1), R(kTwoPi) * nu);
  const R Xe = s.te * fastm::sqrt(R(1.4142135623730951) * s.sth * fastm::div(R(1e3 / kTwoPi) * s.omega0, nu));
  const R lx = fastm::log(Xe);
  const R exm = fastm::exp(-Xe * R(1.0 / 47.2));
  const R fm = R(2.011) * fastm::exp(-fastm::exp(R(1.035) * lx) * R(1.0 / 4.7)) -
               fastm::cos(Xe * R(0.5)) * fastm::exp(-fastm::exp(R(1.2) * lx) * R(1.0 / 2.73)) - R(0.011) * exm +
               (R(0.011) * exm - R(C0) * fastm::exp(R(-8.0 / 3.0) * lx)) * R(0.5) *
                   (R(1) + fastm::tanh(R(10) * (lx - R(LOG120))));
  const R q = s.omega0 * iw;
  const R wpw = s.wp2 * iw;
  R rQ = R(0.5 / cgs::c_light) * wpw * q * q * fm * (s.kr1 + R(6) * s.te) * s.sth * s.sth;
  const R shgm = R(1) - R(0.11) * fastm::log(R(1) + R(0.035) * Xe);
  R rV = R(1.0 / cgs::c_light) * wpw * q * (s.kr0 * shgm) * s.cth;
  // invariant form (nu is the plasma-frame frequency here)
  const R inu = fastm::div(R(1), nu);
  const R js = jscale * inu * inu;
  jI *= js;
  jQ *= js;
  jV *= js;
  aI *= nu;
  aQ *= nu;
  aV *= nu;
  rQ *= nu;
  rV *= nu;
  const R pf = fastm::div(fastm::sqrt(jQ * jQ + jV * jV), jI);
  if (pf > R(1)) {
    const R ipf = fastm::div(R(1), pf + R(0.005));
    jQ *= ipf;
    jV *= ipf;
  }
  c.jI = jI; c.jQ = jQ; c.jV = jV;
  c.aI = aI; c.aQ = aQ; c.aV = aV;
  c.rQ = rQ; c.rV = rV;
  return c;
}

}  // namespace phx
