// CheckFile.hpp -- TEST INFRASTRUCTURE: stand-in for the reference's debug check-file writers,
// which write no numbers that the time step uses.
#pragma once
#include <filesystem>
#include <initializer_list>
#include <string>
template <typename F>
class FieldCheckFile {
 public:
  FieldCheckFile(const char*) {}
  void set_output_filename(const std::filesystem::path&) {}
  void output(std::initializer_list<const F*>) {}
};
template <typename S>
class MeshSelectionCheckFile {
 public:
  MeshSelectionCheckFile(const char*) {}
  void output(const S&) {}
};
template <typename TS>
class TimeSeriesCheckFile {
 public:
  TimeSeriesCheckFile(const char*) {}
  void output(const std::string&) {}
};
