// config.toml + command-line overrides, with the reference's key set and semantics (src/host/io/config.hpp:35-381):
// a TOML subset (sections, key = value, "#" comments outside double quotes, quoted strings), `section.key=value`
// overrides where any camera.frequenc* override first removes every frequency form of the file, typed required and
// optional keys, exactly one frequency form (single, list, linspace, logspace) with duplicates detected by their
// "%e" spelling (they name the HDF5 datasets), and an error for any unknown key.  Error messages are the reference's.
#pragma once

#include <map>
#include <string>
#include <vector>

#include "../../../include/phoenix_b200.h"

namespace phx {

struct RunConfig {
  bool show_header = false;
  std::string outdir;
  std::string image = "hdf5";  // hdf5, text, both or none
  int block_size = 10;         // HDF5 pixels per block side
  std::string dump_file, grid_file;
  bool gpu_decode = false;
  PhxReadOptions read{3, 1, 1, -1};
  PhxRenderParams render{};
  std::vector<double> frequencies;
};

// Throws std::runtime_error("Line N: ...") on malformed input.
void parse_toml(const std::string& text, std::map<std::string, std::string>& kv);

// Reads the frequency form of `kv` into `out` (marks the key used). Throws std::runtime_error.
void read_frequencies(const std::map<std::string, std::string>& kv, std::vector<std::string>& used,
                      std::vector<double>& out);

// Loads `path`, applies the overrides, validates.  Throws std::runtime_error with the reference's messages.
RunConfig load_config(const std::string& path, const std::vector<std::string>& overrides);

}  // namespace phx
