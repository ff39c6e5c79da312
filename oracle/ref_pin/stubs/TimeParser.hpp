// TimeParser.hpp -- TEST INFRASTRUCTURE: stand-in for the reference's time parser; the pin
// driver writes every time as a plain number of seconds, which this parser reads back.
#pragma once
#include <string>
#include "Config.hpp"
template <typename T>
class TimeParser {
 public:
  TimeParser(const Config&) {}
  TimeParser(const TimeParser&, const Config&) {}
  T parse(const std::string& s) const { return s.empty() ? T(0) : T(std::stod(s)); }
};
