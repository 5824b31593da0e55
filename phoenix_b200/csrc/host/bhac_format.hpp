// The BHAC block-AMR dump format as PHOENIX reads it (host/io/bhac_io.hpp:331-499):
//
//   [leaf 0 .. leaf N-1]   each: nwini arrays of nx0*nx1*nx2 doubles (cell = i + j nx0 + k nx0 nx1),
//                          then (nx0+1)(nx1+1)(nx2+1)*nws staggered doubles (skipped by readers)
//   [AMR forest]           one int is_leaf flag per node, pre-order; the 8 children of a refined node in x-fastest
//                          order (child c -> (2i + c%2, 2j + (c/2)%2, 2k + c/4)); base blocks in Morton order of their
//                          (i,j,k) when the snapshot is space-filling-curve ordered, else k-outer / i-inner
//   [nx0 nx1 nx2]          3 ints (cells per block)
//   [neqpar]               neqpar_n doubles (equation parameters: [0] = adiabatic index, [nspin] = spin)
//   [footer, 40 bytes]     ints nleafs, levmax, ndim, ndir, nwini, nws, neqpar_n, it; double t
//
// Leaves appear in the data section in the order the forest walk meets them.
#pragma once

#include <algorithm>
#include <array>
#include <cstdint>
#include <utility>
#include <vector>

namespace phx {
namespace bhac {

// Interleave the low 21 bits of a (bit 3b), b (bit 3b+1) and c (bit 3b+2).
inline uint64_t morton3(uint32_t a, uint32_t b, uint32_t c) {
  uint64_t z = 0;
  for (int bit = 0; bit < 21; bit++) {
    z |= (uint64_t)((a >> bit) & 1u) << (3 * bit);
    z |= (uint64_t)((b >> bit) & 1u) << (3 * bit + 1);
    z |= (uint64_t)((c >> bit) & 1u) << (3 * bit + 2);
  }
  return z;
}

// Base blocks (i, j, k) in the order their sub-forests appear in the dump.
inline std::vector<std::array<int, 3>> base_block_order(const int ng[3], bool sfc) {
  std::vector<std::array<int, 3>> out;
  out.reserve((size_t)ng[0] * ng[1] * ng[2]);
  if (sfc) {
    std::vector<std::pair<uint64_t, std::array<int, 3>>> keyed;
    keyed.reserve((size_t)ng[0] * ng[1] * ng[2]);
    for (int i = 0; i < ng[0]; i++)
      for (int j = 0; j < ng[1]; j++)
        for (int k = 0; k < ng[2]; k++) keyed.push_back({morton3(i, j, k), {i, j, k}});
    std::sort(keyed.begin(), keyed.end(),
              [](const std::pair<uint64_t, std::array<int, 3>>& x, const std::pair<uint64_t, std::array<int, 3>>& y) {
                return x.first < y.first;
              });
    for (auto& e : keyed) out.push_back(e.second);
  } else {
    for (int k = 0; k < ng[2]; k++)
      for (int j = 0; j < ng[1]; j++)
        for (int i = 0; i < ng[0]; i++) out.push_back({i, j, k});
  }
  return out;
}

inline void child_index(int child, int i, int j, int k, int* ci, int* cj, int* ck) {
  *ci = 2 * i + (child & 1);
  *cj = 2 * j + ((child >> 1) & 1);
  *ck = 2 * k + (child >> 2);
}

struct Footer {
  int32_t nleafs, levmax, ndim, ndir, nwini, nws, neqpar_n, it;
  double t;
};
static_assert(sizeof(Footer) == 40, "BHAC footer is 40 bytes");

}  // namespace bhac
}  // namespace phx
