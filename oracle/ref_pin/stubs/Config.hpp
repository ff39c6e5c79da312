// Config.hpp -- TEST INFRASTRUCTURE: stand-in for the reference's configuration header
// (src/Config/Config.hpp, a Boost property tree), placed where the reference includes it when
// oracle/ref_pin builds the reference's hot-path kernels. It holds string key/value pairs; the
// pin driver fills the mesh section ("cell count", "cell size", "origin") so that the
// reference's own Cartesian2DMesh constructor reads its geometry from it. Nothing else of the
// configuration is used on the path. The NIMROD reader's driver sets "bbox" (and reads count()).
#pragma once
#include <array>
#include <cctype>
#include <filesystem>
#include <type_traits>
#include <map>
#include <sstream>
#include <string>
#include <utility>
#include <vector>

namespace stdfs = std::filesystem;

// A section: key/value pairs (kv), its own value (value) and sub-sections in order (children;
// the time-series driver builds "source" / "data" / "transform" sections). Keys compare as
// written. get<bool> reads "true"/"false" as well as numbers, get<char> the first character.
struct ConfigChild;
class Config {
 public:
  std::map<std::string, std::string> kv;
  std::string value;
  std::vector<ConfigChild> children;
  Config() {}
  size_t count(const std::string& key) const;
  template <typename T>
  T get(const std::string& key, const T& def = T()) const {
    auto it = kv.find(key);
    if (it == kv.end()) return def;
    return parse<T>(it->second, def);
  }
  template <typename T>
  T get_value(const T& def = T()) const {
    return value.empty() ? def : parse<T>(value, def);
  }
  // the named sub-section; without one, this section itself (the kernels' pin reads the mesh
  // keys through it) or, when given, `def`
  const Config& get_child(const std::string& key) const;
  const Config& get_child(const std::string& key, const Config& def) const;
  const ConfigChild* begin() const;
  const ConfigChild* end() const;
  std::pair<const ConfigChild*, const ConfigChild*> equal_range(const std::string&) const;

 private:
  template <typename T>
  static T parse(const std::string& s, const T& def) {
    if constexpr (std::is_same<T, std::string>::value) {
      return s;
    } else if constexpr (std::is_same<T, std::filesystem::path>::value) {
      return std::filesystem::path(s);
    } else if constexpr (std::is_same<T, bool>::value) {
      if (s == "true") return true;
      if (s == "false") return false;
      std::istringstream is(s);
      int v = def ? 1 : 0;
      is >> v;
      return v != 0;
    } else if constexpr (std::is_same<T, char>::value) {
      return s.empty() ? def : s[0];
    } else {
      std::istringstream is(s);
      T v = def;
      is >> v;
      return v;
    }
  }
};
struct ConfigChild {
  std::string first;
  Config second;
};
inline size_t Config::count(const std::string& key) const {
  size_t n = kv.count(key);
  for (const ConfigChild& c : children) n += c.first == key ? 1 : 0;
  return n;
}
inline const Config& Config::get_child(const std::string& key) const {
  for (const ConfigChild& c : children)
    if (c.first == key) return c.second;
  return *this;
}
inline const Config& Config::get_child(const std::string& key, const Config& def) const {
  for (const ConfigChild& c : children)
    if (c.first == key) return c.second;
  return def;
}
inline const ConfigChild* Config::begin() const { return children.data(); }
inline const ConfigChild* Config::end() const { return children.data() + children.size(); }
inline std::pair<const ConfigChild*, const ConfigChild*> Config::equal_range(const std::string& key) const {
  // the children with this key, when they are consecutive (as the driver adds them)
  const ConfigChild* b = begin();
  while (b != end() && b->first != key) ++b;
  const ConfigChild* e = b;
  while (e != end() && e->first == key) ++e;
  return {b, e};
}

// boost::algorithm::to_lower_copy, the one string algorithm the time-series reader uses
namespace boost {
namespace algorithm {
inline std::string to_lower_copy(const std::string& s) {
  std::string r = s;
  for (char& ch : r) ch = char(std::tolower(static_cast<unsigned char>(ch)));
  return r;
}
}  // namespace algorithm
}  // namespace boost

// comma-separated numbers, as the reference's split_string reads "nx, ny"
template <typename T, size_t D>
std::array<T, D> split_string(const std::string& in, const char sep = ',') {
  std::array<T, D> out{};
  std::istringstream is(in);
  std::string tok;
  for (size_t i = 0; i < D && std::getline(is, tok, sep); ++i) {
    std::istringstream t(tok);
    t >> out[i];
  }
  return out;
}

class GlobalConfig {
 public:
  Config mesh;
  static GlobalConfig& instance() {
    static GlobalConfig g;
    return g;
  }
  const Config& mesh_configuration() const { return mesh; }
  const Config& boundary_configuration(const std::string&) const { return mesh; }
  const Config& time_series_configuration(const std::string&) const { return mesh; }
  std::vector<std::string> output_files_list() const { return {}; }
  std::filesystem::path simulation_base_path() const { return "."; }
};
