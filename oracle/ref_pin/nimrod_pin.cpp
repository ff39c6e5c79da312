// nimrod_pin.cpp -- TEST INFRASTRUCTURE: runs the reference's own NIMROD raster reader
// (NIMRODRasterFormat, src/Raster/RasterFormats/NIMROD.cpp:313-566) on the CPU so that the
// package's reader (mfcm_b200/raster.py) can be checked against it. Built by
// oracle/ref_pin/build.py into oracle/_ref/libsv_refpin_nimrod.so from the reference's sources;
// only tests/ load it.
//
// The driver constructs the reader on a file, with the configuration's "bbox" key set when a
// bounding box is given, and copies out everything the reader holds: the five header arrays,
// the whole grid as read (buffer_, file order, north row first), the crop's pixel corners, the
// cropped values (values_), the geotransform, the no-data value and the reader's own lower-left
// corner (llc()). The reader keeps these private or protected, so its header is included with
// both read as `public`; the reader's code itself is compiled as the reference wrote it.
#include "sycl.hpp"

#include <array>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "Mesh.hpp"
#include "Cartesian2DMesh.hpp"
#include "Field.hpp"
#include "Config.hpp"
#include "RasterFormat.hpp"

#define private public
#define protected public
#include "NIMROD.hpp"
#undef protected
#undef private
#include "NIMROD.cpp"

namespace {
void put_error(char* err, uint64_t cap, const char* msg) {
  if (err != nullptr && cap > 0) {
    std::snprintf(err, cap, "%s", msg);
  }
}
}  // namespace

extern "C" {

// Reads `path` with NIMRODRasterFormat<double>. bbox: xmin, ymin, xmax, ymax, or null for none.
// Outputs (each may be null):
//   h1[31], h2[28], h3[45], h4[56], h5[51]: the header arrays as read;
//   dims[9]: nxpx, nypx, ulc_xpx, ulc_ypx, lrc_xpx, lrc_ypx, ncols(), nrows(), values_.size();
//   geo[6]: the geotransform; llc[2]: the reader's llc(); nodata[1];
//   buffer (buffer_cap doubles): the whole grid in file order;
//   values (values_cap doubles): values_ (the crop, row-major, north row first).
// Returns 0 when the reader succeeded, 1 when it threw (its message in err), 2 when a capacity
// was too small for what it read.
int refpin_nimrod_read(const char* path, const double* bbox, int16_t* h1, float* h2, float* h3, char* h4,
                       int16_t* h5, uint64_t* dims, double* geo, double* llc, double* nodata, double* buffer,
                       uint64_t buffer_cap, double* values, uint64_t values_cap, char* err, uint64_t err_cap) {
  try {
    Config conf;
    if (bbox != nullptr) {
      char s[160];
      std::snprintf(s, sizeof(s), "%.17g,%.17g,%.17g,%.17g", bbox[0], bbox[1], bbox[2], bbox[3]);
      conf.kv["bbox"] = s;
    }
    NIMRODRasterFormat<double> r(stdfs::path(path), conf);
    if (h1) std::copy(r.h1_.begin(), r.h1_.end(), h1);
    if (h2) std::copy(r.h2_.begin(), r.h2_.end(), h2);
    if (h3) std::copy(r.h3_.begin(), r.h3_.end(), h3);
    if (h4) std::copy(r.h4_.begin(), r.h4_.end(), h4);
    if (h5) std::copy(r.h5_.begin(), r.h5_.end(), h5);
    if (dims) {
      dims[0] = r.nxpx_;
      dims[1] = r.nypx_;
      dims[2] = r.ulc_xpx_;
      dims[3] = r.ulc_ypx_;
      dims[4] = r.lrc_xpx_;
      dims[5] = r.lrc_ypx_;
      dims[6] = r.ncols();
      dims[7] = r.nrows();
      dims[8] = r.values_.size();
    }
    if (geo) std::copy(r.geotrans_.begin(), r.geotrans_.end(), geo);
    if (llc) {
      const std::array<double, 2> c = r.llc();
      llc[0] = c[0];
      llc[1] = c[1];
    }
    if (nodata) nodata[0] = r.nodata_value_;
    if (buffer) {
      if (r.buffer_.size() > buffer_cap) return 2;
      std::copy(r.buffer_.begin(), r.buffer_.end(), buffer);
    }
    if (values) {
      if (r.values_.size() > values_cap) return 2;
      std::copy(r.values_.begin(), r.values_.end(), values);
    }
    return 0;
  } catch (const std::exception& e) {
    put_error(err, err_cap, e.what());
    return 1;
  }
}

}  // extern "C"
