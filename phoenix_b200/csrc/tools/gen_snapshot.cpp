// phx_gen_snapshot: writes a seeded synthetic BHAC block-AMR GRMHD snapshot (dump + grid file) that PHOENIX and this
// library read byte-for-byte the same way.
//
// Spacetime: Kerr, MKS-BHAC coordinates (x1 = ln r on [ln r_min, ln r_max], x2 in [0, pi], x3 in [0, 2 pi]).
// Mesh: blocks of nx^3 cells on a base grid of nxlone cells; a block at level L < nlevels is refined when its centre
//       lies in the torus region (r in [ref_r0, ref_r1], |theta - pi/2| < ref_dth), so the levels nest.
// Fields, all evaluated at the geometric cell centre:
//   rho   constant-angular-momentum torus (inner edge r_in, pressure maximum r_max, l^2 = r_max, enthalpy
//         h = 1/r - l^2 / (2 r^2 sin^2 theta)) to the power 1/(gamma-1), tapered by exp(-(r/r_taper)^2), times
//         log-normal noise exp(sigma z - sigma^2/2), plus a floor 1e-5 r^-1.5
//   u     K rho^gamma / (gamma-1) + floor 1e-7 r^-2.5, with K fixed by the enthalpy normalisation
//   B     curl of A_phi = max(rho_torus - 0.2, 0), scaled so that <p_gas> / <p_mag> = beta over the torus body, plus a weak monopole
//         background b_mono (1 - cos theta) so that no cell has B = 0 (GRMHD snapshots never do)
//   u^i   Keplerian Omega = 1/(R^1.5 + a), R = r sin theta, inside the torus (Eulerian observer outside), with
//         seeded 10% perturbations of each spatial component
// Noise comes from SplitMix64 keyed on (seed, level, global cell coordinates), so it does not depend on block order.
// The primitives are converted to BHAC conserved variables with the metric at the cell centroid, the inverse of the
// decode every reader applies.
#include <omp.h>

#include <cinttypes>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../core/defs.cuh"
#include "../host/bhac_format.hpp"

namespace {

// The generator keeps its own FP64 metric arithmetic (rather than the render headers, which are tuned for the
// kernel) so that the bytes it writes for a given seed never change.
namespace gm {

struct Pt {
  double r, s, c, s2, tp, sig, q;
};

Pt point(double a, double hs, double x1, double x2) {
  Pt p;
  p.r = std::exp(x1);
  const double s2x = std::sin(2.0 * x2), c2x = std::cos(2.0 * x2);
  const double th = x2 + 0.5 * hs * s2x;
  p.tp = 1.0 + hs * c2x;
  p.s = std::sin(th);
  p.c = std::cos(th);
  p.s2 = p.s * p.s;
  p.sig = p.r * p.r + a * a * p.c * p.c;
  p.q = 2.0 * p.r / p.sig;
  return p;
}

struct Cov {
  double tt, t1, t3, x11, x13, x22, x33;
};

Cov cov(const Pt& p, double a) {
  Cov g;
  const double opq = 1.0 + p.q;
  g.tt = p.q - 1.0;
  g.t1 = p.q * p.r;
  g.t3 = -a * p.s2 * p.q;
  g.x11 = opq * p.r * p.r;
  g.x13 = -a * p.s2 * opq * p.r;
  g.x22 = p.sig * p.tp * p.tp;
  g.x33 = p.s2 * (p.sig + a * a * p.s2 * opq);
  return g;
}

struct Contra {
  double tt, t1;
};

Contra contra(const Pt& p) {
  Contra u;
  u.tt = -(1.0 + p.q);
  u.t1 = 2.0 / p.sig;
  return u;
}

// out = g V over the spatial block (V^0 = 0) plus the g_t. column (used for lowering spatial vectors).
void lower(const Cov& g, const double V[4], double out[4]) {
  out[0] = g.tt * V[0] + g.t1 * V[1] + g.t3 * V[3];
  out[1] = g.t1 * V[0] + g.x11 * V[1] + g.x13 * V[3];
  out[2] = g.x22 * V[2];
  out[3] = g.t3 * V[0] + g.x13 * V[1] + g.x33 * V[3];
}

double sqrt_det_gamma(double a, double hs, double x1, double x2) {
  const Cov g = cov(point(a, hs, x1, x2), a);
  return std::sqrt(g.x22 * (g.x11 * g.x33 - g.x13 * g.x13));
}

// Volume-weighted cell centroid (Simpson 1-4-1 per axis), the point every BHAC reader evaluates the metric at.
void centroid(double a, double hs, const double X[3], const double dx[3], double Xbar[3]) {
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

}  // namespace gm

// Conserved slots of the dump (D, S_1..3, tau, B^1..3, D s, then Lorentz factor and xi).
enum { kCD = 0, kCS1 = 1, kCTau = 4, kCB1 = 5, kCDS = 8 };

struct Opts {
  std::string out = ".";
  uint64_t seed = 0;
  int base[3] = {64, 32, 32};
  int nlevels = 3;
  int block = 8;
  int nws = 3;
  int sfc = 1;
  double spin = 0.9375;
  double gam = 13.0 / 9.0;
  double hslope = 0.25;
  double r_min = 1.2, r_max_dom = 1000.0;
  double ref_r0 = 4.0, ref_r1 = 20.0, ref_dth = 0.5;
  double r_in = 6.0, r_pmax = 12.0, r_taper = 40.0;
  double sigma = 0.5;
  double beta = 100.0;
  double vpert = 0.1;
  double bmono = 0.05;
};

uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Standard normal number for (key, stream) by Box-Muller on two SplitMix64 draws.
double gauss(uint64_t key, int stream) {
  const uint64_t h1 = splitmix64(key ^ (0x1000193ull * (2 * stream + 1)));
  const uint64_t h2 = splitmix64(h1 ^ 0xD6E8FEB86659FD93ull);
  const double u1 = ((h1 >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  const double u2 = ((h2 >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  return std::sqrt(-2.0 * std::log(u1)) * std::cos(phx::kTwoPi * u2);
}

struct Leaf {
  int level, i, j, k;
};

struct Gen {
  Opts o;
  double xmin[3], xmax[3];
  int ng[3];
  double K;        // polytropic constant
  double bscale;   // field normalisation
  double hmax;

  double theta_of(double x2) const { return x2 + 0.5 * o.hslope * std::sin(2.0 * x2); }

  // Torus density without noise (normalised to ~1 at the pressure maximum).
  double rho_torus(double r, double th) const {
    const double s = std::sin(th);
    const double l2 = o.r_pmax;
    const double h = 1.0 / r - l2 / (2.0 * r * r * s * s) - (1.0 / o.r_in - l2 / (2.0 * o.r_in * o.r_in));
    if (!(h > 0.0)) return 0.0;
    return std::pow(h / hmax, 1.0 / (o.gam - 1.0)) * std::exp(-(r / o.r_taper) * (r / o.r_taper));
  }

  double aphi(double x1, double x2) const {
    return std::max(rho_torus(std::exp(x1), theta_of(x2)) - 0.2, 0.0);
  }

  // Field B^1, B^2 (unscaled) from the curl of A_phi at (x1, x2).
  void field(double x1, double x2, double* B1, double* B2) const {
    const double d = 1e-5;
    const double r = std::exp(x1), th = theta_of(x2), s = std::sin(th), c = std::cos(th);
    const double tp = 1.0 + o.hslope * std::cos(2.0 * x2);
    const double sqrtg = (r * r + o.spin * o.spin * c * c) * s * r * tp;
    const double dA2 = (aphi(x1, x2 + d) - aphi(x1, x2 - d)) / (2.0 * d);
    const double dA1 = (aphi(x1 + d, x2) - aphi(x1 - d, x2)) / (2.0 * d);
    *B1 = dA2 / sqrtg;
    *B2 = -dA1 / sqrtg;
  }

  void setup() {
    for (int d = 0; d < 3; d++) ng[d] = o.base[d] / o.block;
    xmin[0] = std::log(o.r_min);
    xmax[0] = std::log(o.r_max_dom);
    xmin[1] = 0.0;
    xmax[1] = phx::kPi;
    xmin[2] = 0.0;
    xmax[2] = phx::kTwoPi;
    hmax = 1.0 / o.r_pmax - 0.5 / o.r_pmax - (1.0 / o.r_in - o.r_pmax / (2.0 * o.r_in * o.r_in));
    K = (o.gam - 1.0) * hmax / o.gam;
    // field scale: <p_gas> / <p_mag> = beta averaged over the torus body (rho_torus > 0.2) on a fixed (x1, x2)
    // lattice
    double psum = 0.0, bsum = 0.0;
    for (int ia = 0; ia < 512; ia++) {
      const double x1 = xmin[0] + (ia + 0.5) * (xmax[0] - xmin[0]) / 512;
      for (int ib = 0; ib < 256; ib++) {
        const double x2 = (ib + 0.5) * phx::kPi / 256;
        const double rt = rho_torus(std::exp(x1), theta_of(x2));
        if (!(rt > 0.2)) continue;
        psum += K * std::pow(rt, o.gam);
        double B1, B2;
        field(x1, x2, &B1, &B2);
        const gm::Cov g = gm::cov(gm::point(o.spin, o.hslope, x1, x2), o.spin);
        bsum += 0.5 * (g.x11 * B1 * B1 + g.x22 * B2 * B2);
      }
    }
    bscale = bsum > 0.0 ? std::sqrt(psum / (o.beta * bsum)) : 0.0;
  }

  bool refine(int level, int i, int j, int k) const {
    if (level >= o.nlevels) return false;
    const double sc = 1.0 / (double)(1 << (level - 1));
    const double w0 = (xmax[0] - xmin[0]) / ng[0] * sc, w1 = (xmax[1] - xmin[1]) / ng[1] * sc;
    (void)k;
    const double x1c = xmin[0] + (i + 0.5) * w0, x2c = xmin[1] + (j + 0.5) * w1;
    const double r = std::exp(x1c), th = theta_of(x2c);
    return r >= o.ref_r0 && r <= o.ref_r1 && std::fabs(th - 0.5 * phx::kPi) < o.ref_dth;
  }

  void walk(int level, int i, int j, int k, std::vector<int>& flags, std::vector<Leaf>& leaves) const {
    if (refine(level, i, j, k)) {
      flags.push_back(0);
      for (int ch = 0; ch < 8; ch++) {
        int ci, cj, ck;
        phx::bhac::child_index(ch, i, j, k, &ci, &cj, &ck);
        walk(level + 1, ci, cj, ck, flags, leaves);
      }
    } else {
      flags.push_back(1);
      leaves.push_back({level, i, j, k});
    }
  }

  // Conserved block of one leaf: nwini = 11 arrays of cells doubles.
  void leaf_block(const Leaf& lf, double* out) const {
    const int nx = o.block, cells = nx * nx * nx;
    const double inv_scale = 1.0 / (double)(1 << (lf.level - 1));
    const int ind[3] = {lf.i, lf.j, lf.k};
    double lb[3], dx[3];
    for (int d = 0; d < 3; d++) {
      const double dx1 = (xmax[d] - xmin[d]) / ng[d];
      const double dxc0 = (xmax[d] - xmin[d]) / o.base[d];
      lb[d] = xmin[d] + ind[d] * dx1 * inv_scale;
      dx[d] = dxc0 * inv_scale;
    }
    const double a = o.spin, gam = o.gam;
    for (int cell = 0; cell < cells; cell++) {
      const int ci = cell % nx, cj = (cell / nx) % nx, ck = cell / (nx * nx);
      const double X[3] = {lb[0] + (ci + 0.5) * dx[0], lb[1] + (cj + 0.5) * dx[1], lb[2] + (ck + 0.5) * dx[2]};
      const uint64_t gi = (uint64_t)lf.i * nx + ci, gj = (uint64_t)lf.j * nx + cj, gk = (uint64_t)lf.k * nx + ck;
      const uint64_t key =
          splitmix64(o.seed * 0x2545F4914F6CDD1Dull + ((uint64_t)lf.level << 58) + (gi << 38) + (gj << 19) + gk);
      const double r = std::exp(X[0]), th = theta_of(X[1]);

      // primitives
      const double rt = rho_torus(r, th);
      const double noise = std::exp(o.sigma * gauss(key, 0) - 0.5 * o.sigma * o.sigma);
      const double rho_t = rt * noise;
      const double rho = rho_t + 1e-5 * std::pow(r, -1.5);
      const double uu = K * std::pow(rho_t, gam) / (gam - 1.0) + 1e-7 * std::pow(r, -2.5);
      double B[4] = {0.0, 0.0, 0.0, 0.0};
      field(X[0], X[1], &B[1], &B[2]);
      B[1] *= bscale;
      B[2] *= bscale;
      {
        // monopole background: A_phi = b_mono (1 - cos theta) -> B^1 = b_mono sin(theta) theta' / sqrt(-g)
        const double tp = 1.0 + o.hslope * std::cos(2.0 * X[1]);
        const double c = std::cos(th);
        B[1] += o.bmono / ((r * r + a * a * c * c) * r);
        (void)tp;
      }

      // metric at the centroid (the decode uses the same point)
      double Xb[3];
      gm::centroid(a, o.hslope, X, dx, Xb);
      const gm::Pt p = gm::point(a, o.hslope, Xb[0], Xb[1]);
      const gm::Cov g = gm::cov(p, a);
      const gm::Contra gu = gm::contra(p);
      const double alpha = 1.0 / std::sqrt(-gu.tt);
      const double beta1 = gu.t1 / (-gu.tt);  // shift (beta^2 = beta^3 = 0)

      // u^i = lfac v^i (Eulerian 3-velocity times Lorentz factor)
      double gv[4] = {0.0, 0.0, 0.0, 0.0};
      if (rt > 0.0) {
        const double R = r * std::sin(th);
        const double om = 1.0 / (std::pow(R, 1.5) + a);
        const double nrm = -(g.tt + 2.0 * g.t3 * om + g.x33 * om * om);
        if (nrm > 0.0) {
          const double ut = 1.0 / std::sqrt(nrm);
          gv[1] = ut * beta1;  // U^1 = 0
          gv[3] = om * ut;     // U^3 + U^t beta^3, beta^3 = 0
        }
      }
      double gvd[4];
      gm::lower(g, gv, gvd);
      const double mag = std::sqrt(std::max(gvd[1] * gv[1] + gvd[2] * gv[2] + gvd[3] * gv[3], 0.0));
      for (int d = 1; d <= 3; d++) gv[d] += o.vpert * mag * gauss(key, d);
      gm::lower(g, gv, gvd);
      const double lfac = std::sqrt(1.0 + gvd[1] * gv[1] + gvd[2] * gv[2] + gvd[3] * gv[3]);
      (void)alpha;

      // conserved variables
      const double v[4] = {0.0, gv[1] / lfac, gv[2] / lfac, gv[3] / lfac};
      double vd[4], Bd[4];
      gm::lower(g, v, vd);
      gm::lower(g, B, Bd);
      const double Bsq = Bd[1] * B[1] + Bd[2] * B[2] + Bd[3] * B[3];
      const double Bv = Bd[1] * v[1] + Bd[2] * v[2] + Bd[3] * v[3];
      const double v2 = vd[1] * v[1] + vd[2] * v[2] + vd[3] * v[3];
      const double xi = lfac * lfac * (rho + gam * uu);
      const double press = (gam - 1.0) * uu;
      const double D = rho * lfac;
      double* c = out;
      c[(size_t)kCD * cells + cell] = D;
      for (int d = 1; d <= 3; d++) c[(size_t)(kCS1 + d - 1) * cells + cell] = (xi + Bsq) * vd[d] - Bv * Bd[d];
      c[(size_t)kCTau * cells + cell] = xi - press - D + 0.5 * (Bsq + Bsq * v2 - Bv * Bv);
      for (int d = 1; d <= 3; d++) c[(size_t)(kCB1 + d - 1) * cells + cell] = B[d];
      c[(size_t)kCDS * cells + cell] = D * press / std::pow(rho, gam);
      c[(size_t)9 * cells + cell] = lfac;
      c[(size_t)10 * cells + cell] = xi;
    }
  }
};

void usage() {
  std::fprintf(stderr,
               "usage: phx_gen_snapshot --out DIR [--seed S] [--base N1 N2 N3] [--nlevels L] [--block B] [--nws W]\n"
               "       [--sfc 0|1] [--spin A] [--hslope H] [--refine R0 R1 DTH] [--beta B] [--sigma S] [--bmono B]\n");
}

}  // namespace

int main(int argc, char** argv) {
  Gen G;
  Opts& o = G.o;
  for (int i = 1; i < argc; i++) {
    std::string a = argv[i];
    auto need = [&](int n) {
      if (i + n >= argc) {
        usage();
        std::exit(2);
      }
    };
    if (a == "--out") { need(1); o.out = argv[++i]; }
    else if (a == "--seed") { need(1); o.seed = std::strtoull(argv[++i], nullptr, 10); }
    else if (a == "--base") { need(3); for (int d = 0; d < 3; d++) o.base[d] = std::atoi(argv[++i]); }
    else if (a == "--nlevels") { need(1); o.nlevels = std::atoi(argv[++i]); }
    else if (a == "--block") { need(1); o.block = std::atoi(argv[++i]); }
    else if (a == "--nws") { need(1); o.nws = std::atoi(argv[++i]); }
    else if (a == "--sfc") { need(1); o.sfc = std::atoi(argv[++i]); }
    else if (a == "--spin") { need(1); o.spin = std::atof(argv[++i]); }
    else if (a == "--hslope") { need(1); o.hslope = std::atof(argv[++i]); }
    else if (a == "--beta") { need(1); o.beta = std::atof(argv[++i]); }
    else if (a == "--sigma") { need(1); o.sigma = std::atof(argv[++i]); }
    else if (a == "--bmono") { need(1); o.bmono = std::atof(argv[++i]); }
    else if (a == "--refine") { need(3); o.ref_r0 = std::atof(argv[++i]); o.ref_r1 = std::atof(argv[++i]); o.ref_dth = std::atof(argv[++i]); }
    else { usage(); return 2; }
  }
  for (int d = 0; d < 3; d++) {
    if (o.base[d] <= 0 || o.base[d] % o.block) {
      std::fprintf(stderr, "base grid must be a positive multiple of the block size\n");
      return 2;
    }
  }
  if (o.nlevels < 1 || o.nlevels > 16) {
    std::fprintf(stderr, "nlevels must be in 1..16\n");
    return 2;
  }
  G.setup();

  // forest
  std::vector<int> flags;
  std::vector<Leaf> leaves;
  for (const auto& b : phx::bhac::base_block_order(G.ng, o.sfc != 0)) G.walk(1, b[0], b[1], b[2], flags, leaves);
  int levmax = 1;
  for (const Leaf& l : leaves) levmax = std::max(levmax, l.level);

  const std::string dump_path = o.out + "/dump.dat", grid_path = o.out + "/grid.in";
  FILE* f = std::fopen(dump_path.c_str(), "wb");
  if (!f) {
    std::fprintf(stderr, "cannot create %s\n", dump_path.c_str());
    return 1;
  }
  const int nwini = 11, cells = o.block * o.block * o.block;
  const size_t leaf_doubles = (size_t)nwini * cells;
  const size_t stag_doubles = (size_t)(o.block + 1) * (o.block + 1) * (o.block + 1) * o.nws;
  const int chunk = 1024;
  std::vector<double> buf((size_t)chunk * leaf_doubles);
  std::vector<double> stag(stag_doubles, 0.0);
  for (size_t l0 = 0; l0 < leaves.size(); l0 += chunk) {
    const int nl = (int)std::min<size_t>(chunk, leaves.size() - l0);
#pragma omp parallel for schedule(dynamic, 4)
    for (int q = 0; q < nl; q++) G.leaf_block(leaves[l0 + q], buf.data() + (size_t)q * leaf_doubles);
    for (int q = 0; q < nl; q++) {
      std::fwrite(buf.data() + (size_t)q * leaf_doubles, sizeof(double), leaf_doubles, f);
      if (stag_doubles) std::fwrite(stag.data(), sizeof(double), stag_doubles, f);
    }
  }
  std::fwrite(flags.data(), sizeof(int), flags.size(), f);
  const int nx[3] = {o.block, o.block, o.block};
  std::fwrite(nx, sizeof(int), 3, f);
  const double neqpar[4] = {o.gam, 0.0, 0.0, o.spin};
  std::fwrite(neqpar, sizeof(double), 4, f);
  phx::bhac::Footer ft;
  ft.nleafs = (int32_t)leaves.size();
  ft.levmax = levmax;
  ft.ndim = 3;
  ft.ndir = 3;
  ft.nwini = nwini;
  ft.nws = o.nws;
  ft.neqpar_n = 4;
  ft.it = 0;
  ft.t = 0.0;
  std::fwrite(&ft, sizeof ft, 1, f);
  const bool ok = std::ferror(f) == 0;
  std::fclose(f);
  if (!ok) {
    std::fprintf(stderr, "write error on %s\n", dump_path.c_str());
    return 1;
  }

  FILE* gf = std::fopen(grid_path.c_str(), "w");
  if (!gf) {
    std::fprintf(stderr, "cannot create %s\n", grid_path.c_str());
    return 1;
  }
  std::fprintf(gf, "nxlone1 = %d\nnxlone2 = %d\nnxlone3 = %d\n\n", o.base[0], o.base[1], o.base[2]);
  std::fprintf(gf, "xprobminx1 = %.17g\nxprobminx2 = 0.0\nxprobminx3 = 0.0\n\n", G.xmin[0]);
  std::fprintf(gf, "xprobmax1 = %.17g\nxprobmax2 = 0.5\nxprobmax3 = 1.0\n\n", G.xmax[0]);
  std::fprintf(gf, "hslope = %.17g\n", o.hslope);
  std::fclose(gf);

  std::printf("{\"dump\": \"%s\", \"grid\": \"%s\", \"nleafs\": %zu, \"cells\": %zu, \"levels\": %d, \"seed\": %" PRIu64
              ", \"bytes\": %zu}\n",
              dump_path.c_str(), grid_path.c_str(), leaves.size(), leaves.size() * (size_t)cells, levmax, o.seed,
              leaves.size() * (leaf_doubles + stag_doubles) * 8 + flags.size() * 4 + 12 + 32 + 40);
  return 0;
}
