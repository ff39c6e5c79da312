// ts_pin.cpp -- TEST INFRASTRUCTURE: runs the reference's own time-series reader on the CPU so
// that the deck reader's time series (mfcm_b200/config.py, mfcm_b200.TimeSeries) can be checked
// against it. Built by oracle/ref_pin/build.py into oracle/_ref/libsv_refpin_ts.so from the
// reference's sources; only tests/ load it.
//
// What runs here is the reference's code: TimeSeries<double, double>::load with its inline and
// CSV loaders (src/Input/TimeSeries.cpp:178-285, the CSV through the rapidcsv 8.51 that the
// reference vendors in src/rapidcsv/), its transform, and TimeSeries::at (ts_linterp,
// TimeSeries.cpp:26-47). The configuration is the stand-in of oracle/ref_pin/stubs/Config.hpp,
// and times are plain numbers of seconds (the stand-in time parser reads them with std::stod):
// the reference's own time parser is built on Boost date-time, which is not available.
#include "sycl.hpp"

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <memory>
#include <string>
#include <vector>

#include "DataArray.hpp"
#include "DataArray.cpp"
#include "Config.hpp"
#include "TimeParameters.hpp"
#include "TimeSeries.hpp"
#include "TimeSeries.cpp"

std::shared_ptr<sycl::queue> get_sycl_queue(void) { return std::make_shared<sycl::queue>(); }

namespace {
void put_error(char* err, uint64_t cap, const char* msg) {
  if (err != nullptr && cap > 0) std::snprintf(err, cap, "%s", msg);
}
void fill(Config& c, const char* const* keys, const char* const* vals, int n) {
  for (int i = 0; i < n; ++i) c.kv[keys[i]] = vals[i];
}
}  // namespace

extern "C" {

// TimeSeries<double, double>::load of a "time series" section: its keys (source, filename,
// separator, headers, ...), the inline source's data entries (time, value) when source is
// inline, and the transform section's keys. Up to cap points are copied out; *n gets the
// count. Returns 0, or 1 when the reader threw (its message in err).
int refpin_ts_load(const char* const* keys, const char* const* vals, int nkv, const char* const* dkeys,
                   const char* const* dvals, int ndata, const char* const* tkeys, const char* const* tvals,
                   int ntr, double* times, double* values, uint64_t cap, uint64_t* n, char* err, uint64_t errcap) {
  try {
    Config conf;
    fill(conf, keys, vals, nkv);
    if (ndata > 0) {
      Config source, data;
      for (int i = 0; i < ndata; ++i) {
        Config point;
        point.value = dvals[i];
        data.children.push_back({dkeys[i], point});
      }
      source.children.push_back({"data", data});
      conf.children.push_back({"source", source});
    }
    if (ntr > 0) {
      Config tr;
      fill(tr, tkeys, tvals, ntr);
      conf.children.push_back({"transform", tr});
    }
    TimeParser<double> parser(conf);
    auto ts = TimeSeries<double, double>::load(get_sycl_queue(), parser, conf, false);
    const std::vector<double>& t = ts->get_time_array().host_vector();
    const std::vector<double>& v = ts->get_value_array().host_vector();
    *n = t.size();
    for (size_t i = 0; i < t.size() && i < cap; ++i) {
      times[i] = t[i];
      values[i] = v[i];
    }
    return 0;
  } catch (const std::exception& e) {
    put_error(err, errcap, e.what());
    return 1;
  }
}

// TimeSeries<double, double>::at for the series (t, v) at the query times q (each below the
// last knot: at or beyond it the reference reads past its arrays).
int refpin_ts_at(const double* t, const double* v, uint64_t n, const double* q, uint64_t nq, double* out) {
  try {
    TimeSeries<double, double> ts(get_sycl_queue(), std::vector<double>(t, t + n), std::vector<double>(v, v + n),
                                  false);
    for (uint64_t i = 0; i < nq; ++i) out[i] = ts.at(q[i]);
    return 0;
  } catch (const std::exception& e) {
    std::cerr << "ts_pin: " << e.what() << std::endl;
    return -1;
  }
}

}  // extern "C"
