"""Host checks of the device geometry code (core/*.cuh compiled by g++): the Walker-Penrose constant that the FP32 and
mixed kernels use in place of transporting the polarization vector, and the exact double remainder of the wrap.

Along FP64 geodesics integrated with the kernels' own RK4 (core/geodesic.cuh, F transported as the reference does),
kappa = (r + i a cos) (sin B - i A) stays constant, and cos 2chi / sin 2chi rebuilt from kappa on an observer's screen
pair (core/kerr.cuh wp_components) equal those of the transported F.  The rays dive to r ~ 2-4, cross the equator and
pass within a degree of the pole; the agreement is bounded by the integration error of the transported F itself.
"""
from __future__ import annotations

import os
import subprocess

import pytest

from tests.conftest import ROOT

SRC = r"""
#include <cmath>
#include <cstdio>
#include "geodesic.cuh"
#include "camera.cuh"
using namespace phx;

// One ray: start point (r0, x2), wave vector direction, polarization guess; steps dl = h r until r leaves [rmin, 1e3].
static void ray(double a, double r0, double x2, double k1, double k2, double k3, double h, double rmin) {
  const double hs = 0.25;
  GeoState<double, 12> g;
  double x[4] = {0, std::log(r0), x2, 0.3}, k[4] = {0, k1, k2, k3}, f[4] = {0, 0.01, 0.2, 0.05};
  const KerrPt<double> p = kerr_point(a, hs, x[1], x[2]);
  const Cov<double> c = cov_metric(p, a);
  normalize_null(c, k);
  double kd[4];
  symv(c, k, kd);
  f[0] = -(kd[1] * f[1] + kd[2] * f[2] + kd[3] * f[3]) / kd[0];
  double kap0[2];
  walker_penrose(a, p, k, f, kap0);
  for (int i = 0; i < 4; i++) { g.hi[i] = x[i]; g.hi[4 + i] = k[i]; g.hi[8 + i] = f[i]; }
  for (int i = 0; i < 12; i++) g.lo[i] = 0;
  double drift = 0, evpa = 0, rlo = 1e30, thlo = 10, thhi = -10;
  for (int n = 0; n < 20000; n++) {
    double X[4], K[4], F[4];
    for (int i = 0; i < 4; i++) { X[i] = g.hi[i]; K[i] = g.hi[4 + i]; F[i] = g.hi[8 + i]; }
    const KerrPt<double> q = kerr_point(a, hs, X[1], X[2]);
    const Cov<double> cc = cov_metric(q, a);
    double kap[2];
    walker_penrose(a, q, K, F, kap);
    const double m = std::hypot(kap0[0], kap0[1]);
    drift = std::fmax(drift, std::hypot(kap[0] - kap0[0], kap[1] - kap0[1]) / m);
    rlo = std::fmin(rlo, q.r);
    const double th = std::atan2(q.s, q.c);
    thlo = std::fmin(thlo, th);
    thhi = std::fmax(thhi, th);
    if (cc.tt < -1e-3) {  // a static observer exists: compare the two EVPA routes on its screen
      double U[4] = {1.0 / std::sqrt(-cc.tt), 0, 0, 0};
      const double b[4] = {0.0, 0.3, 1.0 / q.tp, 0.2};
      double perp[4], para[4], om, Fd[4], C2, S2;
      observer_axes(cc, sqrt_neg_g(q), K, U, b, perp, para, &om);
      symv(cc, F, Fd);
      const double C1 = dot4(Fd, perp), S1 = dot4(Fd, para);
      wp_components(a, q, K, perp, para, kap0, &C2, &S2);
      const double n1 = C1 * C1 + S1 * S1, n2 = C2 * C2 + S2 * S2;
      evpa = std::fmax(evpa, std::fabs((C1 * C1 - S1 * S1) / n1 - (C2 * C2 - S2 * S2) / n2));
      evpa = std::fmax(evpa, std::fabs(2 * C1 * S1 / n1 - 2 * C2 * S2 / n2));
    }
    rk4_step<double, false, 12>(a, hs, g, h * q.r);
    const double rn = std::exp(g.hi[1]);
    if (rn < rmin || rn > 1e3) break;
  }
  std::printf("%.3e %.3e %.4f %.4f %.4f\n", drift, evpa, rlo, thlo, thhi);
}

int main() {
  ray(0.9375, 40.0, 0.9, -0.02, 0.0021, 0.0012, 0.002, 1.5);    // dives to r ~ 3.8, into the south, back out
  ray(0.5, 20.0, 1.4, -0.05, -0.0040, 0.0030, 0.002, 1.5);      // heads north and plunges through the horizon
  ray(0.99, 30.0, 0.12, -0.03, -0.0015, 0.0004, 0.002, 1.5);    // starts 7 deg from the pole and passes over it
  ray(0.9375, 12.0, 1.6, -0.04, 0.0002, 0.0070, 0.001, 2.05);   // grazes the photon region near the horizon
  return 0;
}
"""


@pytest.fixture(scope="module")
def wp_results(tmp_path_factory):
    d = tmp_path_factory.mktemp("wp")
    src, exe = d / "wp.cpp", d / "wp"
    src.write_text(SRC)
    core = os.path.join(ROOT, "phoenix_b200", "csrc", "core")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-I" + core, str(src), "-o", str(exe)])
    out = subprocess.check_output([str(exe)]).decode().split("\n")
    return [[float(v) for v in line.split()] for line in out if line.strip()]


def test_walker_penrose_constant_is_conserved(wp_results):
    for drift, _, rlo, thlo, thhi in wp_results:
        assert rlo < 6.0  # every ray reaches the strong-field region
        assert drift <= 1e-7, (drift, rlo)


def test_evpa_from_walker_penrose_matches_transport(wp_results):
    for _, evpa, *_ in wp_results:
        assert evpa <= 1e-7, evpa
    # the set covers both hemispheres and a polar passage
    assert min(r[3] for r in wp_results) < 0.2 and max(r[4] for r in wp_results) > 1.7


FMOD_SRC = r"""
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <initializer_list>
#include "defs.cuh"

static uint64_t bits(double v) { uint64_t b; std::memcpy(&b, &v, 8); return b; }

int main() {
  const double ys[2] = {phx::kPi, phx::kTwoPi};
  uint64_t s = 0x9E3779B97F4A7C15ull, n = 0, bad = 0;
  auto next = [&]() { s ^= s << 13; s ^= s >> 7; s ^= s << 17; return s; };
  for (double y : ys) {
    for (int i = 0; i < 2000000; i++) {
      const uint64_t u = next();
      double x;
      if (i % 4 == 0) {  // within a few ulps of a multiple of y
        const double m = (double)((int64_t)(u % 401) - 200) * y;
        x = std::nextafter(m, (u >> 20) & 1 ? 1e300 : -1e300);
        for (int k = (int)((u >> 21) % 4); k > 0; k--) x = std::nextafter(x, (u >> 23) & 1 ? 1e300 : -1e300);
      } else {
        x = ((double)(u >> 11) / 9007199254740992.0 - 0.5) * 1400.0 / (1 + (u % 7));
      }
      n++;
      if (bits(phx::fmod_exact(x, y)) != bits(std::fmod(x, y))) bad++;
    }
    for (double x : {0.0, -0.0, y, -y, 2 * y, -3 * y, std::nextafter(y, 0.0), std::nextafter(-y, 0.0)}) {
      n++;
      if (bits(phx::fmod_exact(x, y)) != bits(std::fmod(x, y))) bad++;
    }
  }
  std::printf("%llu %llu\n", (unsigned long long)n, (unsigned long long)bad);
  return 0;
}
"""


def test_fmod_exact_matches_fmod_bit_for_bit(tmp_path):
    """The device's double remainder (core/defs.cuh fmod_exact) against the C library's fmod, bit for bit: random
    arguments up to 700 in magnitude and arguments within a few ulps of multiples of pi and 2 pi."""
    src, exe = tmp_path / "fm.cpp", tmp_path / "fm"
    src.write_text(FMOD_SRC)
    core = os.path.join(ROOT, "phoenix_b200", "csrc", "core")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I" + core, str(src), "-o", str(exe)])
    n, bad = map(int, subprocess.check_output([str(exe)]).decode().split())
    assert n > 4_000_000 and bad == 0, (n, bad)


SHIFT_SRC = r"""
#include <cmath>
#include <cstdio>
#include "geodesic.cuh"
using namespace phx;

// The mixed kernel's FP64 geodesic steps (kShift: stage trig shifted from the step start, Newton-refined reciprocals)
// against the direct evaluation at every stage with exact divisions, for states near the horizon and at the step
// sizes taken there; and, as the scale of what rounding alone does, the direct step from a start point moved by one
// ulp in x1 and x2.
int main() {
  uint64_t s = 0x2545F4914F6CDD1Dull;
  auto u01 = [&]() { s ^= s << 13; s ^= s >> 7; s ^= s << 17; return (double)(s >> 11) / 9007199254740992.0; };
  double worst = 0, ulp = 0;
  int n = 0;
  for (int i = 0; i < 20000; i++) {
    const double a = 0.5 + 0.49 * u01(), hs = 0.25;
    const double r = 1.6 + 3.0 * u01(), x2 = 0.05 + 3.0 * u01();
    double k[4] = {0, (u01() - 0.5) * 0.5, (u01() - 0.5) * 0.3, (u01() - 0.5) * 0.4};
    const KerrPt<double> p = kerr_point(a, hs, std::log(r), x2);
    normalize_null(cov_metric(p, a), k);
    if (!std::isfinite(k[0])) continue;
    GeoState<double, 8> g1, g2, g3;
    const double x[4] = {0, std::log(r), x2, 1.0};
    for (int j = 0; j < 4; j++) { g1.hi[j] = x[j]; g1.hi[4 + j] = k[j]; }
    for (int j = 0; j < 8; j++) g1.lo[j] = 0;
    g2 = g1;
    g3 = g1;
    g3.hi[1] = std::nextafter(g3.hi[1], 1e9);
    g3.hi[2] = std::nextafter(g3.hi[2], 1e9);
    const double dt = -(0.0005 + 0.01 * u01()) * r;  // stage offsets within the short series (|dx| < 0.025)
    rk4_step<double, false, 8, false>(a, hs, g1, dt);
    rk4_step<double, false, 8, true>(a, hs, g2, dt);
    rk4_step<double, false, 8, false>(a, hs, g3, dt);
    for (int j = 0; j < 8; j++) {
      if (j == 1 || j == 2) continue;  // the components moved by hand
      const double sc = std::fmax(std::fabs(g1.hi[j]), 1e-3);
      worst = std::fmax(worst, std::fabs(g1.hi[j] - g2.hi[j]) / sc);
      ulp = std::fmax(ulp, std::fabs(g1.hi[j] - g3.hi[j]) / sc);
    }
    n++;
  }
  std::printf("%d %.3e %.3e\n", n, worst, ulp);
  return 0;
}
"""


def test_shifted_island_stages_match_direct(tmp_path):
    """The mixed geodesic's shifted stages stay within what one ulp of the start point does to the direct step."""
    src, exe = tmp_path / "sh.cpp", tmp_path / "sh"
    src.write_text(SHIFT_SRC)
    core = os.path.join(ROOT, "phoenix_b200", "csrc", "core")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-I" + core, str(src), "-o", str(exe)])
    n, worst, ulp = subprocess.check_output([str(exe)]).decode().split()
    assert int(n) > 15000, n
    assert float(worst) <= float(ulp) and float(worst) <= 1e-11, (worst, ulp)


RCP_SRC = r"""
#include <cmath>
#include <cstdio>
#include <cstdint>
#include "defs.cuh"

int main() {
  uint64_t s = 0x9E3779B97F4A7C15ull;
  auto u01 = [&]() { s ^= s << 13; s ^= s >> 7; s ^= s << 17; return (double)(s >> 11) / 9007199254740992.0; };
  double worst = 0;
  int n = 0;
  for (int i = 0; i < 4000000; i++) {
    const double x = (u01() < 0.5 ? -1 : 1) * std::exp((u01() - 0.5) * 2 * 69.0);  // |x| in [1e-30, 1e30]
    const double r = phx::fastm::rcp_nr(x), q = 1.0 / x;
    const double ulps = std::fabs(r - q) / (std::nextafter(std::fabs(q), 1e308) - std::fabs(q));
    worst = std::fmax(worst, ulps);
    n++;
  }
  const double edge[] = {0.0, -0.0, 1e-300, 1e300, -1e-40, 1e40, INFINITY};
  int bad_edge = 0;
  for (double x : edge) {
    const double r = phx::fastm::rcp_nr(x), q = 1.0 / x;
    if (!(r == q || (std::isnan(r) && std::isnan(q)))) bad_edge++;
  }
  std::printf("%d %.3f %d\n", n, worst, bad_edge);
  return 0;
}
"""


def test_newton_reciprocal_within_an_ulp(tmp_path):
    """The mixed geodesic's FP64 reciprocal (core/defs.cuh rcp_nr: float seed, two Newton-Raphson steps) against the
    IEEE quotient 1/x: within one ulp over |x| in [1e-30, 1e30], and exactly the quotient outside that range."""
    src, exe = tmp_path / "rcp.cpp", tmp_path / "rcp"
    src.write_text(RCP_SRC)
    core = os.path.join(ROOT, "phoenix_b200", "csrc", "core")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I" + core, str(src), "-o", str(exe)])
    n, worst, bad_edge = subprocess.check_output([str(exe)]).decode().split()
    assert int(n) == 4000000 and float(worst) <= 1.0 and int(bad_edge) == 0, (n, worst, bad_edge)
