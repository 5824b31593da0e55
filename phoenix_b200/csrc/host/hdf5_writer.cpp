// Minimal HDF5 writer (see hdf5_writer.hpp).  File layout, every structure 8-byte aligned:
//   superblock v0 | root object header | local heap header + names | B-tree node | symbol-table nodes |
//   dataset object headers | dataset data
#include "hdf5_writer.hpp"

#include <algorithm>
#include <cstdio>
#include <cstring>

namespace phx {

namespace {

constexpr uint64_t kUndef = ~0ull;
constexpr int kLeafK = 4;       // symbol-table node holds 2 * 4 entries
constexpr int kInternalK = 16;  // B-tree node holds 2 * 16 children
constexpr size_t kSuperblock = 96;
constexpr size_t kSymEntry = 40;
constexpr size_t kSnodSize = 8 + 2 * kLeafK * kSymEntry;
constexpr size_t kBtreeSize = 24 + (2 * kInternalK + 1) * 8 + 2 * kInternalK * 8;

size_t pad8(size_t n) { return (n + 7) & ~size_t(7); }

struct Buf {
  std::vector<uint8_t> b;
  void at(size_t off, const void* p, size_t n) {
    if (b.size() < off + n) b.resize(off + n, 0);
    std::memcpy(b.data() + off, p, n);
  }
  void u8(size_t off, uint8_t v) { at(off, &v, 1); }
  void u16(size_t off, uint16_t v) { at(off, &v, 2); }
  void u32(size_t off, uint32_t v) { at(off, &v, 4); }
  void u64(size_t off, uint64_t v) { at(off, &v, 8); }
};

// One version-1 object-header message at `off`: type, data size (multiple of 8), flags; returns the next offset.
size_t message(Buf& f, size_t off, uint16_t type, const std::vector<uint8_t>& data, uint8_t flags) {
  const size_t n = pad8(data.size());
  f.u16(off, type);
  f.u16(off + 2, (uint16_t)n);
  f.u8(off + 4, flags);
  std::vector<uint8_t> d(data);
  d.resize(n, 0);
  if (n) f.at(off + 8, d.data(), n);
  return off + 8 + n;
}

template <class T>
void put(std::vector<uint8_t>& v, T x) {
  const uint8_t* p = reinterpret_cast<const uint8_t*>(&x);
  v.insert(v.end(), p, p + sizeof(T));
}

}  // namespace

bool write_hdf5(const std::string& path, std::vector<H5Dataset> ds, std::string* err) {
  auto fail = [&](const std::string& m) {
    if (err) *err = m;
    return false;
  };
  if (ds.empty()) return fail("no datasets");
  std::sort(ds.begin(), ds.end(), [](const H5Dataset& a, const H5Dataset& b) { return std::strcmp(a.name.c_str(), b.name.c_str()) < 0; });
  for (size_t i = 1; i < ds.size(); i++)
    if (ds[i].name == ds[i - 1].name) return fail("duplicate dataset name " + ds[i].name);
  for (const auto& d : ds)
    if (d.name.empty() || d.data.size() != d.rows * d.cols) return fail("bad dataset " + d.name);
  const size_t nsnod = (ds.size() + 2 * kLeafK - 1) / (2 * kLeafK);
  if (nsnod > 2 * kInternalK) return fail("too many datasets for one B-tree node");

  // local heap data segment: "" at 0, then the names (each NUL-terminated, padded to 8), then one free block
  std::vector<uint8_t> heap(8, 0);
  std::vector<uint64_t> name_off;
  for (const auto& d : ds) {
    name_off.push_back(heap.size());
    heap.insert(heap.end(), d.name.begin(), d.name.end());
    heap.resize(pad8(heap.size() + 1), 0);
  }
  const uint64_t free_off = heap.size();
  put<uint64_t>(heap, 1);   // next free block: none (the library's end-of-list value)
  put<uint64_t>(heap, 16);  // size of this free block

  // addresses
  const size_t root_hdr = kSuperblock;
  const size_t root_hdr_size = 16 + 8 + 16;
  const size_t heap_hdr = root_hdr + root_hdr_size;
  const size_t heap_data = heap_hdr + 32;
  const size_t btree = pad8(heap_data + heap.size());
  const size_t snod0 = btree + kBtreeSize;
  const size_t dshdr0 = snod0 + nsnod * kSnodSize;
  const size_t dshdr_size = 16 + (8 + 8) + (8 + 24) + (8 + 24) + (8 + 24);
  size_t data_at = dshdr0 + ds.size() * dshdr_size;
  std::vector<size_t> data_off;
  for (const auto& d : ds) {
    data_off.push_back(data_at);
    data_at = pad8(data_at + d.data.size() * sizeof(double));
  }
  const size_t eof = data_at;

  Buf f;
  f.b.reserve(eof);
  // superblock version 0
  static const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
  f.at(0, sig, 8);
  f.u8(8, 0);   // superblock version
  f.u8(9, 0);   // free-space storage version
  f.u8(10, 0);  // root group symbol table entry version
  f.u8(11, 0);
  f.u8(12, 0);  // shared header message format version
  f.u8(13, 8);  // size of offsets
  f.u8(14, 8);  // size of lengths
  f.u8(15, 0);
  f.u16(16, kLeafK);
  f.u16(18, kInternalK);
  f.u32(20, 0);  // file consistency flags
  f.u64(24, 0);  // base address
  f.u64(32, kUndef);
  f.u64(40, eof);
  f.u64(48, kUndef);
  // root group symbol table entry (cache type 1: B-tree and heap addresses in the scratch pad)
  f.u64(56, 0);
  f.u64(64, root_hdr);
  f.u32(72, 1);
  f.u32(76, 0);
  f.u64(80, btree);
  f.u64(88, heap_hdr);

  // root object header: one symbol-table message
  f.u8(root_hdr, 1);
  f.u8(root_hdr + 1, 0);
  f.u16(root_hdr + 2, 1);
  f.u32(root_hdr + 4, 1);
  f.u32(root_hdr + 8, (uint32_t)(root_hdr_size - 16));
  {
    std::vector<uint8_t> m;
    put<uint64_t>(m, btree);
    put<uint64_t>(m, heap_hdr);
    message(f, root_hdr + 16, 0x0011, m, 1);
  }

  // local heap
  f.at(heap_hdr, "HEAP", 4);
  f.u8(heap_hdr + 4, 0);
  f.u64(heap_hdr + 8, heap.size());
  f.u64(heap_hdr + 16, free_off);
  f.u64(heap_hdr + 24, heap_data);
  f.at(heap_data, heap.data(), heap.size());

  // B-tree node (group, leaf level): key i = heap offset of the last name in child i-1 (key 0: "")
  f.at(btree, "TREE", 4);
  f.u8(btree + 4, 0);
  f.u8(btree + 5, 0);
  f.u16(btree + 6, (uint16_t)nsnod);
  f.u64(btree + 8, kUndef);
  f.u64(btree + 16, kUndef);
  f.u64(btree + 24, 0);
  for (size_t c = 0; c < nsnod; c++) {
    const size_t last = std::min(ds.size(), (c + 1) * 2 * kLeafK) - 1;
    f.u64(btree + 32 + 16 * c, snod0 + c * kSnodSize);
    f.u64(btree + 40 + 16 * c, name_off[last]);
  }
  f.at(btree + kBtreeSize - 1, "\0", 1);

  // symbol-table nodes
  for (size_t c = 0; c < nsnod; c++) {
    const size_t at = snod0 + c * kSnodSize;
    const size_t first = c * 2 * kLeafK, last = std::min(ds.size(), first + 2 * kLeafK);
    f.at(at, "SNOD", 4);
    f.u8(at + 4, 1);
    f.u8(at + 5, 0);
    f.u16(at + 6, (uint16_t)(last - first));
    for (size_t e = first; e < last; e++) {
      const size_t ent = at + 8 + (e - first) * kSymEntry;
      f.u64(ent, name_off[e]);
      f.u64(ent + 8, dshdr0 + e * dshdr_size);
      f.u32(ent + 16, 0);
    }
    f.at(at + kSnodSize - 1, "\0", 1);
  }

  // dataset object headers
  for (size_t e = 0; e < ds.size(); e++) {
    const size_t at = dshdr0 + e * dshdr_size;
    f.u8(at, 1);
    f.u8(at + 1, 0);
    f.u16(at + 2, 4);
    f.u32(at + 4, 1);
    f.u32(at + 8, (uint32_t)(dshdr_size - 16));
    size_t p = at + 16;
    // fill value (version 2): allocation late, write if set, no fill value defined
    p = message(f, p, 0x0005, {2, 2, 2, 0}, 1);
    // datatype: IEEE little-endian float64 (class 1, version 1)
    {
      std::vector<uint8_t> m = {0x11, 0x20, 0x3f, 0x00};
      put<uint32_t>(m, 8);
      put<uint16_t>(m, 0);   // bit offset
      put<uint16_t>(m, 64);  // precision
      m.push_back(52);       // exponent location
      m.push_back(11);       // exponent size
      m.push_back(0);        // mantissa location
      m.push_back(52);       // mantissa size
      put<uint32_t>(m, 1023);
      p = message(f, p, 0x0003, m, 1);
    }
    // dataspace (version 1): rank 2, no maximum dimensions
    {
      std::vector<uint8_t> m = {1, 2, 0, 0, 0, 0, 0, 0};
      put<uint64_t>(m, ds[e].rows);
      put<uint64_t>(m, ds[e].cols);
      p = message(f, p, 0x0001, m, 0);
    }
    // layout (version 3): contiguous
    {
      std::vector<uint8_t> m = {3, 1};
      put<uint64_t>(m, data_off[e]);
      put<uint64_t>(m, ds[e].data.size() * sizeof(double));
      p = message(f, p, 0x0008, m, 1);
    }
  }
  for (size_t e = 0; e < ds.size(); e++)
    if (!ds[e].data.empty()) f.at(data_off[e], ds[e].data.data(), ds[e].data.size() * sizeof(double));
  f.b.resize(eof, 0);

  FILE* fp = std::fopen(path.c_str(), "wb");
  if (!fp) return fail("cannot create " + path);
  const bool ok = std::fwrite(f.b.data(), 1, f.b.size(), fp) == f.b.size();
  return std::fclose(fp) == 0 && ok ? true : fail("write error on " + path);
}

}  // namespace phx
