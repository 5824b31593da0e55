// Host-side BHAC reader and decoder (see snapshot.hpp).
#include "snapshot.hpp"

#include <omp.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <memory>
#include <sstream>
#include <stdexcept>

#include "../core/decode.cuh"
#include "bhac_format.hpp"

namespace phx {

namespace {

struct FileCloser {
  void operator()(FILE* f) const {
    if (f) std::fclose(f);
  }
};
using FilePtr = std::unique_ptr<FILE, FileCloser>;

template <class T>
bool read1(FILE* f, T* v) {
  return std::fread(v, sizeof(T), 1, f) == 1;
}

// Pre-order forest walk; leaves appended in file order.
void read_forest_node(FILE* f, int level, int i, int j, int k, std::vector<int32_t>& lev, std::vector<int32_t>& ind,
                      bool& ok) {
  if (!ok) return;
  int32_t is_leaf = 0;
  if (!read1(f, &is_leaf)) {
    ok = false;
    return;
  }
  if (is_leaf) {
    lev.push_back(level);
    ind.push_back(i);
    ind.push_back(j);
    ind.push_back(k);
    return;
  }
  for (int ch = 0; ch < 8; ch++) {
    int ci, cj, ck;
    bhac::child_index(ch, i, j, k, &ci, &cj, &ck);
    read_forest_node(f, level + 1, ci, cj, ck, lev, ind, ok);
  }
}

}  // namespace

void read_grid_file(const std::string& path, int nxlone[3], double xprobmin[3], double xprobmax[3], double* hslope) {
  std::ifstream in(path);
  if (!in) throw std::runtime_error("cannot open grid file " + path);
  std::vector<double> v;
  std::string line;
  while (std::getline(in, line)) {
    std::istringstream ss(line);
    std::string tok, last;
    while (ss >> tok) last = tok;
    if (!last.empty()) v.push_back(std::atof(last.c_str()));
  }
  if (v.size() < 10)
    throw std::runtime_error(path + ": expected 10 lines (nxlone x3, xprobmin x3, xprobmax x3, hslope)");
  for (int d = 0; d < 3; d++) {
    nxlone[d] = (int)v[d];
    xprobmin[d] = v[3 + d];
    xprobmax[d] = v[6 + d];
  }
  *hslope = v[9];
  if (nxlone[0] <= 0 || nxlone[1] <= 0 || nxlone[2] <= 0 || xprobmax[0] <= xprobmin[0] ||
      xprobmax[1] <= xprobmin[1] || xprobmax[2] <= xprobmin[2])
    throw std::runtime_error(path + ": nxlone / xprobmin / xprobmax not set (or empty domain)");
}

std::vector<int32_t> flatten_level_maps(const std::vector<std::vector<int32_t>>& maps, const int32_t ng[3],
                                        int nlevels) {
  const int top = nlevels - 1;
  const size_t f0 = (size_t)ng[0] << top, f1 = (size_t)ng[1] << top, f2 = (size_t)ng[2] << top;
  std::vector<int32_t> flat(f0 * f1 * f2, -1);
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < (long long)f0; i++)
    for (size_t j = 0; j < f1; j++)
      for (size_t k = 0; k < f2; k++) {
        int32_t leaf = -1;
        for (int L = 0; L < nlevels && leaf < 0; L++) {
          const int sh = top - L;
          const size_t d1 = (size_t)ng[1] << L, d2 = (size_t)ng[2] << L;
          leaf = maps[L][(((size_t)i >> sh) * d1 + (j >> sh)) * d2 + (k >> sh)];
        }
        flat[((size_t)i * f1 + j) * f2 + k] = leaf;
      }
  return flat;
}

HostSnapshot load_bhac_meta(const std::string& dump, const std::string& grid, const SnapshotOptions& opt) {
  HostSnapshot s;
  double xmin[3], xmax[3];
  read_grid_file(grid, s.nxlone, xmin, xmax, &s.hslope);

  FilePtr fp(std::fopen(dump.c_str(), "rb"));
  FILE* f = fp.get();
  if (!f) throw std::runtime_error("Can't open " + dump);

  // footer: the last 40 bytes, then nx[3] and the equation parameters just before it
  bhac::Footer ft;
  if (std::fseek(f, -(long)sizeof ft, SEEK_END) != 0 || !read1(f, &ft))
    throw std::runtime_error("Bad read in the dump header. Is " + dump + " a BHAC dump?");
  if (ft.ndim != 3) throw std::runtime_error("Only 3D dumps are supported! (ndim = " + std::to_string(ft.ndim) + ")");
  if (ft.nleafs <= 0 || ft.nwini < 3 || ft.nws < 0 || ft.neqpar_n <= 0)
    throw std::runtime_error("Bad read in the dump header. Is " + dump + " a BHAC dump?");
  std::vector<double> neqpar(ft.neqpar_n);
  bool ok = std::fseek(f, -(long)(sizeof ft + 3 * sizeof(int32_t) + ft.neqpar_n * sizeof(double)), SEEK_END) == 0;
  for (int d = 0; d < 3; d++) ok = ok && read1(f, &s.nx[d]);
  for (int i = 0; i < ft.neqpar_n; i++) ok = ok && read1(f, &neqpar[i]);
  if (!ok || opt.nspin < 0 || opt.nspin >= ft.neqpar_n)
    throw std::runtime_error("Short read in the dump header! (wrong grmhd.nspin?)");
  s.nleafs = ft.nleafs;
  s.nwini = ft.nwini;
  s.nws = ft.nws;
  s.a = neqpar[opt.nspin];
  if (std::fabs(s.a) > 1.0) throw std::runtime_error("Spin " + std::to_string(s.a) + " unphysical (wrong grmhd.nspin?)");
  s.gam = neqpar[0];
  for (int d = 1; d < 3; d++) {
    xmin[d] *= 2.0 * kPi;
    xmax[d] *= 2.0 * kPi;
  }
  if (s.nx[0] <= 0 || s.nx[1] <= 0 || s.nx[2] <= 0) throw std::runtime_error("bad block size in the dump header");
  s.cells = s.nx[0] * s.nx[1] * s.nx[2];
  for (int d = 0; d < 3; d++) {
    if (s.nxlone[d] % s.nx[d] != 0)
      throw std::runtime_error("nxlone[" + std::to_string(d) + "] = " + std::to_string(s.nxlone[d]) +
                               " is not a multiple of the dump's block size " + std::to_string(s.nx[d]) +
                               ": wrong grid file");
    s.ng[d] = s.nxlone[d] / s.nx[d];
    s.x_lo[d] = xmin[d];
    s.x_hi[d] = xmax[d];
  }

  // forest
  const long long leaf_bytes = (long long)s.cells * s.nwini * 8;
  const long long stag_bytes = (long long)(s.nx[0] + 1) * (s.nx[1] + 1) * (s.nx[2] + 1) * s.nws * 8;
  if (std::fseek(f, (long)((long long)s.nleafs * (leaf_bytes + stag_bytes)), SEEK_SET) != 0)
    throw std::runtime_error("short read in the tree (wrong nxlone / grmhd.sfc for this dump?)");
  ok = true;
  for (const auto& b : bhac::base_block_order(s.ng, opt.sfc))
    read_forest_node(f, 1, b[0], b[1], b[2], s.leaf_level, s.leaf_index, ok);
  if (!ok) throw std::runtime_error("short read in the tree (wrong nxlone / grmhd.sfc for this dump?)");
  if ((int)s.leaf_level.size() != s.nleafs)
    throw std::runtime_error("grid mismatch: tree has " + std::to_string(s.leaf_level.size()) +
                             " leaves, header says " + std::to_string(s.nleafs) + " (grmhd.sfc / grid file?)");

  // leaf geometry
  s.lb.resize(3 * (size_t)s.nleafs);
  s.dxc.resize(3 * (size_t)s.nleafs);
  double dx1[3], dxc0[3];
  for (int d = 0; d < 3; d++) {
    dx1[d] = (xmax[d] - xmin[d]) / s.ng[d];
    dxc0[d] = (xmax[d] - xmin[d]) / s.nxlone[d];
  }
  int deepest = 1;
  for (int l = 0; l < s.nleafs; l++) {
    const int lev = s.leaf_level[l];
    if (lev < 1 || lev > kMaxLevels) throw std::runtime_error("leaf level out of range in the forest");
    deepest = std::max(deepest, lev);
    const double inv_scale = 1.0 / (double)(1 << (lev - 1));
    for (int d = 0; d < 3; d++) {
      s.lb[3 * (size_t)l + d] = xmin[d] + s.leaf_index[3 * (size_t)l + d] * dx1[d] * inv_scale;
      s.dxc[3 * (size_t)l + d] = dxc0[d] * inv_scale;
    }
  }

  // per-level leaf maps
  s.nlevels = opt.nlevels == -1 ? deepest : opt.nlevels;
  if (s.nlevels < 1 || s.nlevels > kMaxLevels)
    throw std::runtime_error(std::to_string(s.nlevels) + " AMR levels unsupported (max 16)");
  s.level_map.resize(s.nlevels);
  for (int L = 0; L < s.nlevels; L++) {
    const size_t d0 = (size_t)s.ng[0] << L, d1 = (size_t)s.ng[1] << L, d2 = (size_t)s.ng[2] << L;
    s.level_map[L].assign(d0 * d1 * d2, -1);
    for (int l = 0; l < s.nleafs; l++) {
      if (s.leaf_level[l] - 1 != L) continue;
      const long long i = s.leaf_index[3 * (size_t)l], j = s.leaf_index[3 * (size_t)l + 1],
                      k = s.leaf_index[3 * (size_t)l + 2];
      if (i < 0 || i >= (long long)d0 || j < 0 || j >= (long long)d1 || k < 0 || k >= (long long)d2) continue;
      s.level_map[L][((size_t)i * d1 + j) * d2 + k] = l;
    }
  }

  return s;
}

void stream_leaf_blocks(const std::string& dump, const HostSnapshot& s, int chunk,
                        const std::function<double*(int, int)>& next_buffer,
                        const std::function<void(int, int, const double*)>& ready) {
  FilePtr fp(std::fopen(dump.c_str(), "rb"));
  FILE* f = fp.get();
  if (!f) throw std::runtime_error("Can't open " + dump);
  const size_t leaf_doubles = (size_t)s.nwini * s.cells;
  const long long stag_bytes = (long long)(s.nx[0] + 1) * (s.nx[1] + 1) * (s.nx[2] + 1) * s.nws * 8;
  for (int l0 = 0; l0 < s.nleafs; l0 += chunk) {
    const int nl = std::min(chunk, s.nleafs - l0);
    double* buf = next_buffer(l0, nl);
    for (int q = 0; q < nl; q++) {
      if (std::fread(buf + (size_t)q * leaf_doubles, sizeof(double), leaf_doubles, f) != leaf_doubles)
        throw std::runtime_error("short read in the data, leaf " + std::to_string(l0 + q));
      if (stag_bytes && std::fseek(f, (long)stag_bytes, SEEK_CUR) != 0)
        throw std::runtime_error("short read in the data, leaf " + std::to_string(l0 + q));
    }
    ready(l0, nl, buf);
  }
}

HostSnapshot load_bhac(const std::string& dump, const std::string& grid, const SnapshotOptions& opt) {
  HostSnapshot s = load_bhac_meta(dump, grid, opt);
  // decode: stream the leaf blocks, conserved -> primitive per cell in parallel
  const size_t leaf_doubles = (size_t)s.nwini * s.cells;
  const size_t nprim = (size_t)s.nleafs * s.cells * kNPrim;
  s.prim_f32.assign(nprim, 0.0f);
  if (opt.keep_f64) s.prim_f64.assign(nprim, 0.0);
  const int chunk = 256;
  std::vector<double> raw((size_t)chunk * leaf_doubles);
  stream_leaf_blocks(
      dump, s, chunk, [&](int, int) { return raw.data(); },
      [&](int l0, int nl, const double* buf) {
#pragma omp parallel for schedule(dynamic, 1)
        for (int q = 0; q < nl; q++) {
          const size_t l = (size_t)l0 + q;
          for (int cell = 0; cell < s.cells; cell++) {
            double p[kNPrim];
            cons_to_prim(s.a, s.hslope, s.gam, opt.bpol, s.nwini, s.nx, &s.lb[3 * l], &s.dxc[3 * l],
                         buf + (size_t)q * leaf_doubles, cell, p);
            const size_t o = (l * s.cells + cell) * kNPrim;
            for (int v = 0; v < kNPrim; v++) s.prim_f32[o + v] = (float)p[v];
            if (opt.keep_f64)
              for (int v = 0; v < kNPrim; v++) s.prim_f64[o + v] = p[v];
          }
        }
      });
  return s;
}

}  // namespace phx
