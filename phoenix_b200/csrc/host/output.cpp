// Output writers (see output.hpp).
#include "output.hpp"

#include <cmath>
#include <cstdio>

#include "../core/defs.cuh"
#include "hdf5_writer.hpp"

namespace phx {

namespace {

double unit_length(const PhxRenderParams& p) { return cgs::g_newton * p.mass * cgs::m_sun / cgs::c_light / cgs::c_light; }

double solid_angle(const PhxRenderParams& p) {
  const double d = p.distance * cgs::kpc, L = unit_length(p);
  return (p.fov_x / p.img_width * L / d) * (p.fov_y / p.img_height * L / d);
}

// Impact parameters of pixel (i, j) without the position-angle rotation (the image axes).
void impact(const PhxRenderParams& p, int i, int j, double* a, double* b) {
  *a = -0.5 * p.fov_x + (i + 0.5) * p.fov_x / p.img_width;
  *b = -0.5 * p.fov_y + (j + 0.5) * p.fov_y / p.img_height;
}

const PhxFreqOut& at(const PhxRenderParams& p, const std::vector<PhxFreqOut>& res, int i, int j, int f) {
  return res[((size_t)i * p.img_height + j) * p.nfreqs + f];
}

}  // namespace

void compute_spec(const PhxRenderParams& p, const std::vector<PhxFreqOut>& res, int f, double S[4]) {
  const double dOmega = solid_angle(p);
  for (int q = 0; q < 4; q++) S[q] = 0.0;
  for (int i = 0; i < p.img_width; i++)
    for (int j = 0; j < p.img_height; j++) {
      const PhxFreqOut& r = at(p, res, i, j, f);
      if (!std::isfinite(r.IQUV[0] + r.IQUV[1] + r.IQUV[2] + r.IQUV[3])) continue;
      for (int q = 0; q < 4; q++) S[q] += r.IQUV[q] * dOmega;
    }
  for (int q = 0; q < 4; q++) S[q] *= cgs::jansky;
}

void compute_tau(const PhxRenderParams& p, const std::vector<PhxFreqOut>& res, int f, double T[2]) {
  double s0 = 0.0, s1 = 0.0;
  size_t n = 0;
  for (int i = 0; i < p.img_width; i++)
    for (int j = 0; j < p.img_height; j++) {
      const PhxFreqOut& r = at(p, res, i, j, f);
      if (!std::isfinite(r.IQUV[0] + r.IQUV[1] + r.IQUV[2] + r.IQUV[3] + r.tau + r.tauF)) continue;
      s0 += r.tau;
      s1 += r.tauF;
      n++;
    }
  T[0] = n ? s0 / (double)n : 0.0;
  T[1] = n ? s1 / (double)n : 0.0;
}

bool write_image_text(const std::string& path, const PhxRenderParams& p, const std::vector<PhxFreqOut>& res, int f) {
  FILE* fp = std::fopen(path.c_str(), "w");
  if (!fp) return false;
  const double unit = cgs::jansky * solid_angle(p);
  const double arcsec = 206265.0 * unit_length(p) / (p.distance * cgs::kpc);
  for (int i = 0; i < p.img_width; i++)
    for (int j = 0; j < p.img_height; j++) {
      double a, b;
      impact(p, i, j, &a, &b);
      const PhxFreqOut& r = at(p, res, i, j, f);
      std::fprintf(fp, "%+.15e\t%+.15e\t%+.15e\t%+.15e\t%+.15e\t%+.15e\t%+.15e\t%+.15e\n", a * arcsec, b * arcsec,
                   r.IQUV[0] * unit, r.IQUV[1] * unit, r.IQUV[2] * unit, r.IQUV[3] * unit, r.tau, r.tauF);
    }
  return std::fclose(fp) == 0;
}

bool write_spectrum(const std::string& path, const PhxRenderParams& p, const std::vector<PhxFreqOut>& res) {
  FILE* fp = std::fopen(path.c_str(), "w");
  if (!fp) return false;
  for (int f = 0; f < p.nfreqs; f++) {
    double S[4], T[2];
    compute_spec(p, res, f, S);
    compute_tau(p, res, f, T);
    std::fprintf(fp, "%+.15e\t%+.15e\t%+.15e\t%+.15e\t%+.15e\t%+.15e\t%+.15e\n", p.frequencies[f], S[0], S[1], S[2],
                 S[3], T[0], T[1]);
  }
  return std::fclose(fp) == 0;
}

bool write_image_hdf5(const std::string& path, const PhxRenderParams& p, int bs, const std::vector<PhxFreqOut>& res,
                      std::string* err) {
  if (bs < 1 || p.img_width % bs || p.img_height % bs) {
    if (err) {
      char b[160];
      std::snprintf(b, sizeof b, "output.block_size %d must divide the image size %dx%d", bs, p.img_width,
                    p.img_height);
      *err = b;
    }
    return false;
  }
  const int nbj = p.img_height / bs, nblocks = (p.img_width / bs) * nbj, npb = bs * bs;
  enum { kI, kQ, kU, kV, kTau, kTauF, kAlpha, kBeta };
  auto value = [&](int what, int f, int i, int j) {
    if (what <= kV) return at(p, res, i, j, f).IQUV[what] * cgs::jansky;
    if (what == kTau) return at(p, res, i, j, f).tau;
    if (what == kTauF) return at(p, res, i, j, f).tauF;
    double a, b;
    impact(p, i, j, &a, &b);
    return what == kAlpha ? a : b;
  };
  auto make = [&](const std::string& name, int what, int f) {
    H5Dataset d;
    d.name = name;
    d.rows = nblocks;
    d.cols = npb;
    d.data.resize((size_t)nblocks * npb);
    for (int b = 0; b < nblocks; b++)
      for (int q = 0; q < npb; q++)
        d.data[(size_t)b * npb + q] = value(what, f, (b / nbj) * bs + q / bs, (b % nbj) * bs + q % bs);
    return d;
  };
  std::vector<H5Dataset> ds;
  for (int f = 0; f < p.nfreqs; f++) {
    char fb[64];
    std::snprintf(fb, sizeof fb, "%e", p.frequencies[f]);
    const std::string fs = fb;
    ds.push_back(make("I" + fs, kI, f));
    ds.push_back(make("tau" + fs, kTau, f));
    ds.push_back(make("Q" + fs, kQ, f));
    ds.push_back(make("U" + fs, kU, f));
    ds.push_back(make("V" + fs, kV, f));
    ds.push_back(make("tauF" + fs, kTauF, f));
  }
  ds.push_back(make("alpha", kAlpha, 0));
  ds.push_back(make("beta", kBeta, 0));
  return write_hdf5(path, std::move(ds), err);
}

}  // namespace phx
