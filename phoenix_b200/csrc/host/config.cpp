// config.toml reader: a line lexer for the TOML subset, a declarative table of the typed keys with one generic
// reader over it, and the frequency forms.  Key names, defaults, override rules and message texts follow the
// reference (src/host/io/config.hpp:61-381); see config.hpp.
#include "config.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iterator>
#include <set>
#include <stdexcept>
#include <string_view>
#include <variant>

namespace phx {

namespace {

using KeyValues = std::map<std::string, std::string>;

// Every key that selects or spells a frequency form starts with this (an override of one replaces them all).
constexpr std::string_view kFrequencyFamily = "camera.frequenc";

std::string_view strip(std::string_view s, std::string_view blanks = " \t\r") {
  const size_t first = s.find_first_not_of(blanks);
  if (first == std::string_view::npos) return {};
  return s.substr(first, s.find_last_not_of(blanks) - first + 1);
}

bool in_family(std::string_view key) { return key.substr(0, kFrequencyFamily.size()) == kFrequencyFamily; }

// The part of a line before its comment: the first '#' preceded by an even number of '"' (i.e. not inside a
// double-quoted run).
std::string_view before_comment(std::string_view line) {
  for (size_t hash = line.find('#'); hash != std::string_view::npos; hash = line.find('#', hash + 1)) {
    if (std::count(line.begin(), line.begin() + hash, '"') % 2 == 0) return line.substr(0, hash);
  }
  return line;
}

[[noreturn]] void line_error(int line_no, const std::string& what) {
  throw std::runtime_error("Line " + std::to_string(line_no) + ": " + what);
}

// ---- typed keys ------------------------------------------------------------------------------------------------

// Where a key's value goes.  Numbers are read leniently (atof, integers truncated from the real value), booleans are
// "true" or "1"; an empty numeric or boolean value leaves the default in place.
using Slot = std::variant<bool*, double*, int32_t*, std::string*>;

struct KeySpec {
  const char* name;
  bool required;
  Slot slot;
};

struct Assign {
  const std::string& text;
  void operator()(std::string* s) const { *s = text; }
  void operator()(double* d) const {
    if (!text.empty()) *d = std::atof(text.c_str());
  }
  void operator()(int32_t* i) const {
    if (!text.empty()) *i = (int32_t)std::atof(text.c_str());
  }
  void operator()(bool* b) const {
    if (!text.empty()) *b = text == "true" || text == "1";
  }
};

// Reads table entries from the key/value map; records what it consumed and which required keys were absent.
class TableReader {
 public:
  explicit TableReader(const KeyValues& kv) : kv_(kv) {}

  void read(const KeySpec& k) {
    const auto hit = kv_.find(k.name);
    if (hit == kv_.end()) {
      if (k.required) missing_ += std::string(" ") + k.name;
      return;
    }
    consumed_.emplace_back(k.name);
    std::visit(Assign{hit->second}, k.slot);
  }

  std::vector<std::string>& consumed() { return consumed_; }
  const std::string& missing() const { return missing_; }

 private:
  const KeyValues& kv_;
  std::vector<std::string> consumed_;
  std::string missing_;
};

// ---- frequency forms -------------------------------------------------------------------------------------------

enum class FreqForm { kSingle, kList, kLinspace, kLogspace };

struct FormKey {
  FreqForm form;
  const char* name;
};
constexpr FormKey kFormKeys[] = {{FreqForm::kSingle, "camera.frequency"},
                                 {FreqForm::kList, "camera.frequency_list"},
                                 {FreqForm::kLinspace, "camera.frequency_linspace"},
                                 {FreqForm::kLogspace, "camera.frequency_logspace"}};

double to_number(const std::string& key, std::string_view token) {
  const std::string t(token);
  char* end = nullptr;
  const double v = std::strtod(t.c_str(), &end);
  if (end == t.c_str() || *end != '\0') throw std::runtime_error(key + ": not a number: " + t);
  return v;
}

// The numbers between the first '[' and the last ']' of `text`, comma separated; empty items (a trailing comma) are
// skipped.
std::vector<double> bracket_list(const std::string& key, const std::string& text) {
  const size_t open = text.find('['), close = text.rfind(']');
  if (open == std::string::npos || close == std::string::npos || close < open)
    throw std::runtime_error(key + " must be a list on ONE line: [a, b, ...]");
  const std::string_view inner = std::string_view(text).substr(open + 1, close - open - 1);
  std::vector<double> values;
  size_t from = 0;
  while (from <= inner.size()) {
    const size_t comma = std::min(inner.find(',', from), inner.size());
    const std::string_view item = strip(inner.substr(from, comma - from), " \t");
    if (!item.empty()) values.push_back(to_number(key, item));
    from = comma + 1;
  }
  return values;
}

// n points from start to stop, evenly (linspace) or geometrically (logspace) spaced; the last is `stop` itself.
std::vector<double> spaced(const std::string& key, const std::vector<double>& args, bool geometric) {
  if (args.size() != 3)
    throw std::runtime_error(key + " has " + std::to_string(args.size()) + "arguments! (Expected 3)");
  const double start = args[0], stop = args[1], count = args[2];
  if (!(count >= 2.0 && count <= 1e6) || count != std::floor(count))
    throw std::runtime_error(key + ": n must be an integer >= 2! (use frequency = nu for a single frequency)");
  if (!(start > 0.0) || !(stop > start)) throw std::runtime_error(key + ": need 0 < start < stop!");
  const int n = (int)count;
  const double span = stop - start, ratio = stop / start;
  std::vector<double> nu(n, stop);
  for (int i = 0; i + 1 < n; i++) {
    const double t = double(i) / (n - 1);
    nu[i] = geometric ? start * std::pow(ratio, t) : start + span * t;
  }
  return nu;
}

void check_frequencies(const std::vector<double>& nu) {
  std::set<std::string> names;
  for (const double v : nu) {
    if (!(v > 0.0) || !std::isfinite(v)) throw std::runtime_error("frequencies must be positive and finite");
    char name[64];
    std::snprintf(name, sizeof name, "%e", v);
    if (!names.insert(name).second)
      throw std::runtime_error(std::string("duplicate frequency ") + name +
                               " (they are used to name the HDF5 datasets)");
  }
}

// ---- overrides -------------------------------------------------------------------------------------------------

void apply_overrides(KeyValues& kv, const std::vector<std::string>& overrides) {
  std::vector<std::pair<std::string, std::string>> pairs;
  for (const std::string& arg : overrides) {
    const size_t eq = arg.find('=');
    if (eq == std::string::npos) throw std::runtime_error("Override must be section.key=value: " + arg);
    pairs.emplace_back(arg.substr(0, eq), arg.substr(eq + 1));
  }
  const bool new_frequencies =
      std::any_of(pairs.begin(), pairs.end(), [](const auto& p) { return in_family(p.first); });
  if (new_frequencies) {
    for (auto it = kv.begin(); it != kv.end();) it = in_family(it->first) ? kv.erase(it) : std::next(it);
  }
  for (auto& p : pairs) kv[p.first] = std::move(p.second);
}

// The typed keys of a run, in the order their absence is reported.  The frequency forms are read separately.
std::vector<KeySpec> key_table(RunConfig& c, bool* sfc) {
  PhxRenderParams& p = c.render;
  return {
      {"visual.show_header", true, &c.show_header},
      {"black_hole.mass", true, &p.mass},
      {"black_hole.distance", true, &p.distance},
      {"integration.stepsize", true, &p.stepsize},
      {"integration.max_steps", true, &p.max_steps},
      {"integration.horizon_margin", true, &p.horizon_margin},
      {"integration.max_order", true, &p.max_order},
      {"camera.inclination", true, &p.inclination},
      {"camera.img_width", true, &p.img_width},
      {"camera.img_height", true, &p.img_height},
      {"camera.fov_x", true, &p.fov_x},
      {"camera.fov_y", true, &p.fov_y},
      {"camera.r_cam", true, &p.r_cam},
      {"camera.t_init", true, &p.t_init},
      {"camera.pa", false, &p.pa},
      {"camera.phi", false, &p.phi},
      {"output.dir", true, &c.outdir},
      {"output.image", false, &c.image},
      {"output.block_size", false, &c.block_size},
      {"grmhd.dump_file", true, &c.dump_file},
      {"grmhd.grid_file", true, &c.grid_file},
      {"grmhd.gpu_decode", true, &c.gpu_decode},
      {"grmhd.nspin", true, &c.read.nspin},
      {"grmhd.sfc", true, sfc},
      {"grmhd.nlevels", true, &c.read.nlevels},
      {"grmhd.bpol", true, &c.read.bpol},
      {"plasma.m_unit", true, &p.m_unit},
      {"plasma.r_low", true, &p.r_low},
      {"plasma.r_high", true, &p.r_high},
      {"plasma.sigma_cut", true, &p.sigma_cut},
      {"plasma.thetae_min", true, &p.thetae_min},
      {"plasma.thetae_max", true, &p.thetae_max},
      {"plasma.rt_outer", true, &p.rt_outer},
      {"plasma.beta_c", false, &p.beta_c},
  };
}

}  // namespace

KeyValues parse_toml(const std::string& text) {
  KeyValues kv;
  std::string section;
  const std::string_view all(text);
  int line_no = 0;
  for (size_t at = 0; at < all.size();) {
    const size_t eol = std::min(all.find('\n', at), all.size());
    const std::string_view body = strip(before_comment(all.substr(at, eol - at)));
    at = eol + 1;
    line_no++;
    if (body.empty()) continue;
    if (body.front() == '[') {
      if (body.back() != ']') line_error(line_no, "bad section header");
      section = std::string(strip(body.substr(1, body.size() - 2)));
      continue;
    }
    const size_t eq = body.find('=');
    if (eq == std::string_view::npos) line_error(line_no, "expected key = value");
    std::string_view value = strip(body.substr(eq + 1));
    if (value.size() >= 2 && value.front() == '"' && value.back() == '"') value = value.substr(1, value.size() - 2);
    const std::string_view key = strip(body.substr(0, eq));
    std::string name = section.empty() ? std::string(key) : section + "." + std::string(key);
    if (!kv.emplace(name, std::string(value)).second) line_error(line_no, "duplicate key " + name);
  }
  return kv;
}

std::vector<double> read_frequencies(const KeyValues& kv, std::vector<std::string>& consumed) {
  const FormKey* chosen = nullptr;
  int present = 0;
  for (const FormKey& f : kFormKeys) {
    if (kv.count(f.name)) {
      present++;
      chosen = &f;
    }
  }
  if (present != 1) throw std::runtime_error("Too many (or no) frequency forms given!");
  const std::string key = chosen->name;
  const std::string& text = kv.at(key);
  consumed.push_back(key);
  std::vector<double> nu;
  switch (chosen->form) {
    case FreqForm::kSingle:
      nu = {to_number(key, text)};
      break;
    case FreqForm::kList:
      nu = bracket_list(key, text);
      if (nu.empty()) throw std::runtime_error(key + " is empty!");
      break;
    case FreqForm::kLinspace:
    case FreqForm::kLogspace:
      nu = spaced(key, bracket_list(key, text), chosen->form == FreqForm::kLogspace);
      break;
  }
  check_frequencies(nu);
  return nu;
}

RunConfig load_config(const std::string& path, const std::vector<std::string>& overrides) {
  std::ifstream file(path);
  if (!file) throw std::runtime_error("Cannot open file " + path + ". Perhaps it's a malformed TOML key-value pair?");
  const std::string text((std::istreambuf_iterator<char>(file)), std::istreambuf_iterator<char>());
  KeyValues kv = parse_toml(text);
  apply_overrides(kv, overrides);

  RunConfig c;
  phx_default_params(&c.render);
  c.render.pa = 0.0;  // optional keys and their defaults
  c.render.phi = 0.0;
  c.render.beta_c = 1.0;
  bool sfc = c.read.sfc != 0;
  TableReader reader(kv);
  for (const KeySpec& k : key_table(c, &sfc)) reader.read(k);
  c.read.sfc = sfc ? 1 : 0;

  auto fail = [&](const std::string& what) { throw std::runtime_error(path + ": " + what); };
  try {
    c.frequencies = read_frequencies(kv, reader.consumed());
  } catch (const std::exception& e) {
    fail(e.what());
  }
  if (c.frequencies.size() > (size_t)PHX_MAX_FREQS)
    fail("at most " + std::to_string(PHX_MAX_FREQS) + " frequencies (PHX_MAX_FREQS), got " +
         std::to_string(c.frequencies.size()));
  c.render.nfreqs = (int32_t)c.frequencies.size();
  std::copy(c.frequencies.begin(), c.frequencies.end(), c.render.frequencies);

  static const std::set<std::string> kImageKinds = {"hdf5", "text", "both", "none"};
  if (!kImageKinds.count(c.image)) fail("output.image must be hdf5, text, both or none");
  if (c.block_size < 1) fail("output.block_size must be >= 1");
  if (!(c.render.beta_c > 0.0)) fail("plasma.beta_c must be > 0");
  if (!reader.missing().empty()) fail("missing required key(s):" + reader.missing());
  const std::vector<std::string>& used = reader.consumed();
  for (const auto& entry : kv)
    if (std::find(used.begin(), used.end(), entry.first) == used.end()) fail("unknown key " + entry.first);
  return c;
}

}  // namespace phx
