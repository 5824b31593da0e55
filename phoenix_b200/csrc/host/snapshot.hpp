// Host-side BHAC snapshot: reading the dump + grid file and decoding it (C++17, OpenMP), and the flattened leaf map
// the device sampler uses.  Follows the reference reader (host/io/bhac_io.hpp:143-499): grid file = last token of
// each line (nxlone x3, xprobmin x3, xprobmax x3, hslope; x2 and x3 bounds in units of 2 pi), footer at the end of
// the dump, forest walk in Morton or k-j-i order of base blocks, leaf origins and cell sizes from the level and
// index of each leaf, per-level leaf maps, conserved -> primitive decode at the cell centroid.
#pragma once

#include <cstdint>
#include <functional>
#include <string>
#include <vector>

namespace phx {

struct SnapshotOptions {
  int nspin = 3;     // index of the spin in the dump's equation parameters
  int bpol = 1;      // sign of the poloidal field
  int nlevels = -1;  // AMR levels of the leaf map (-1: the deepest level found)
  bool sfc = true;   // base blocks stored along the Morton curve
  bool keep_f64 = false;  // also keep FP64 primitives (for FP64 renders)
};

struct HostSnapshot {
  int32_t nleafs = 0, nlevels = 0, cells = 0, nwini = 0, nws = 0;
  int32_t nx[3] = {0, 0, 0}, ng[3] = {0, 0, 0}, nxlone[3] = {0, 0, 0};
  double a = 0, hslope = 0, gam = 0;
  double x_lo[3] = {0, 0, 0}, x_hi[3] = {0, 0, 0};  // (x1, x2, x3) domain, x2/x3 in radians
  std::vector<double> lb, dxc;                        // [nleafs][3]
  std::vector<int32_t> leaf_level, leaf_index;        // level (1-based) and (i,j,k) of each leaf
  std::vector<float> prim_f32;                        // [nleafs][cells][8]
  std::vector<double> prim_f64;                       // optional
  std::vector<std::vector<int32_t>> level_map;        // per level, [ng0<<L][ng1<<L][ng2<<L]
};

// Throws std::runtime_error with the reference's messages on malformed input.
void read_grid_file(const std::string& path, int nxlone[3], double xprobmin[3], double xprobmax[3], double* hslope);
HostSnapshot load_bhac(const std::string& dump, const std::string& grid, const SnapshotOptions& opt);

// The reader without the cell data: header, forest, leaf geometry and level maps (prim_* left empty).
HostSnapshot load_bhac_meta(const std::string& dump, const std::string& grid, const SnapshotOptions& opt);

// Streams the leaves' conserved blocks (nwini arrays of `cells` doubles per leaf, staggered fields skipped) in chunks
// of at most `chunk` leaves.  next_buffer(l0, nl) returns where chunk [l0, l0 + nl) is read to (room for nl blocks);
// ready(l0, nl, buf) is called once it holds them.
void stream_leaf_blocks(const std::string& dump, const HostSnapshot& s, int chunk,
                        const std::function<double*(int, int)>& next_buffer,
                        const std::function<void(int, int, const double*)>& ready);

// Finest-level leaf map: slot (i,j,k) of level nlevels-1 holds the first leaf found walking the per-level maps from
// the coarsest level (what the reference's find_leaf_map returns for any point in that slot).
std::vector<int32_t> flatten_level_maps(const std::vector<std::vector<int32_t>>& maps, const int32_t ng[3],
                                        int nlevels);

}  // namespace phx
