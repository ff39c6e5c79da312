// Config.hpp -- TEST INFRASTRUCTURE: stand-in for the reference's configuration header
// (src/Config/Config.hpp, a Boost property tree), placed where the reference includes it when
// oracle/ref_pin builds the reference's hot-path kernels. It holds string key/value pairs; the
// pin driver fills the mesh section ("cell count", "cell size", "origin") so that the
// reference's own Cartesian2DMesh constructor reads its geometry from it. Nothing else of the
// configuration is used on the path. The NIMROD reader's driver sets "bbox" (and reads count()).
#pragma once
#include <array>
#include <filesystem>
#include <map>
#include <sstream>
#include <string>
#include <utility>
#include <vector>

namespace stdfs = std::filesystem;

struct ConfigChild;
class Config {
 public:
  std::map<std::string, std::string> kv;
  Config() {}
  size_t count(const std::string& key) const { return kv.count(key); }
  template <typename T>
  T get(const std::string& key, const T& def = T()) const {
    auto it = kv.find(key);
    if (it == kv.end()) return def;
    std::istringstream is(it->second);
    T v = def;
    is >> v;
    return v;
  }
  template <typename T>
  T get_value(const T& def = T()) const {
    return def;
  }
  const Config& get_child(const std::string&) const { return *this; }
  // sub-sections (none: the hot path reads no configured boundaries or selections)
  const ConfigChild* begin() const;
  const ConfigChild* end() const;
  std::pair<const ConfigChild*, const ConfigChild*> equal_range(const std::string&) const;
};
struct ConfigChild {
  std::string first;
  Config second;
};
inline const ConfigChild* Config::begin() const { return nullptr; }
inline const ConfigChild* Config::end() const { return nullptr; }
inline std::pair<const ConfigChild*, const ConfigChild*> Config::equal_range(const std::string&) const {
  return {nullptr, nullptr};
}
template <>
inline std::string Config::get<std::string>(const std::string& key, const std::string& def) const {
  auto it = kv.find(key);
  return it == kv.end() ? def : it->second;
}

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
  std::vector<std::string> output_files_list() const { return {}; }
  std::filesystem::path simulation_base_path() const { return "."; }
};
