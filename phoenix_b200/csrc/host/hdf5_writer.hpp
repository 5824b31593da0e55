// Minimal HDF5 writer: one file holding 2-D float64 datasets in the root group, in the classic file format
// (HDF5 File Format Specification 3.0: superblock version 0, root group as a symbol table -- a version-1 B-tree of
// symbol-table nodes plus a local heap of names -- and version-1 object headers with dataspace, IEEE little-endian
// float64 datatype, fill-value and contiguous-layout messages).  Readable by any HDF5 library (h5py, RAPTOR's
// rapplot.py).  PHOENIX writes its image dump this way (src/host/io/output.hpp:111-167) through libhdf5, which this
// project does not depend on.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace phx {

struct H5Dataset {
  std::string name;
  uint64_t rows = 0, cols = 0;
  std::vector<double> data;  // rows * cols, row-major
};

// At most 256 datasets (one B-tree node of 32 symbol-table nodes of 8 entries).  Returns false and sets *err on
// failure.
bool write_hdf5(const std::string& path, std::vector<H5Dataset> datasets, std::string* err);

}  // namespace phx
