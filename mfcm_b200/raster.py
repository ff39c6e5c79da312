"""NIMROD raster input (the Met Office radar and model grid format) mapped onto a solver mesh.

The file layout follows the reference's reader (src/Raster/RasterFormats/NIMROD.cpp:313-566),
all big-endian:

- a 4-byte record length of 512, then the header: 31 int16, 28 float32, 45 float32, 56 chars,
  51 int16 (h1 .. h5), then the record length again;
- a 4-byte record length, the nrows x ncols values (h1[15] rows, h1[16] columns, the north
  row first), then the same record length again;
- the value type from h1[11] and its size from h1[12]: 0 = float32 (4 bytes), 1 = int16 or
  int32 (2 or 4 bytes), 2 = signed char (1 byte); the no-data value is h2[6] for float data,
  h1[24] otherwise;
- only the top-left grid origin (h1[23] = 0) is read; the first pixel centre is at easting
  h2[4], northing h2[2], with column and row intervals h2[5] and h2[3].

As in the reference, the values are taken as stored: no-data values stay in the field and the
header's scale factor and offset (h2[7], h2[8]) are not applied (`NimrodRaster.header` has
them).

The reference's raster path cannot deliver a raster to a field. These bugs are fixed here:

- the raster mesh is built with zero cells (Cartesian2DMesh.cpp:71-73 copies the cell counts
  instead of binding them), and from {rows, columns} where the mesh wants {columns, rows}
  (RasterFormat.hpp:78);
- without a bounding box no values are kept (NIMROD.cpp:491-496);
- with one, the mesh keeps the whole file's lower-left corner instead of the crop's (the
  reader's own `llc()`, NIMROD.hpp:60-66, is never used), and a lower-right row past the file
  is clamped to row 0 instead of the last row (NIMROD.cpp:483);
- the values are in file order, north row first, on a mesh whose row 0 is the south row;
- the mapping writes the value at the selection's position instead of the cell's index, and
  skips destination cells whose index exceeds the raster's cell count
  (FieldOperators.hpp:104-114).

Here the raster is a field on its own mesh with row 0 to the south. A solver cell takes the
value of the raster cell containing its centre. This is Cartesian2DMesh::
get_nearest_object_index, Cartesian2DMesh.hpp:179-188, with the same coordinate arithmetic.
Cells whose centre is outside the raster keep their previous value.
"""
import struct

import numpy as np

_H1, _H2, _H3, _H4, _H5 = 31, 28, 45, 56, 51
_HEADER_FMT = f">{_H1}h{_H2}f{_H3}f{_H4}s{_H5}h"
assert struct.calcsize(_HEADER_FMT) == 512

_DTYPES = {(0, 4): ">f4", (1, 2): ">i2", (1, 4): ">i4", (2, 1): ">i1"}


class RasterError(ValueError):
    pass


class NimrodRaster:
    """A NIMROD grid read from a file, optionally cropped to a bounding box.

    Attributes: `values` (nrows x ncols, FP64, row 0 = the southern row), `x0`, `y0` (lower-left
    corner of the kept area), `dx`, `dy` (pixel size), `nodata`, `header` (h1 .. h5)."""

    def __init__(self, path, bbox=None):
        with open(path, "rb") as f:
            data = f.read()
        self._parse(data, bbox)

    @classmethod
    def from_bytes(cls, data, bbox=None):
        r = cls.__new__(cls)
        r._parse(data, bbox)
        return r

    def _parse(self, data, bbox):
        if bbox is not None:
            bbox = [float(b) for b in bbox]
            if len(bbox) != 4:
                raise RasterError("a bounding box has four numbers: xmin ymin xmax ymax")
            if bbox[2] <= bbox[0]:
                raise RasterError(f"bounding box has negative x-dimension: {bbox[2]} <= {bbox[0]}")
            if bbox[3] <= bbox[1]:
                raise RasterError(f"bounding box has negative y-dimension: {bbox[3]} <= {bbox[1]}")
        pos = 0

        def u32():
            nonlocal pos
            if pos + 4 > len(data):
                raise RasterError(f"could not read 4 bytes at offset {pos}")
            (v,) = struct.unpack_from(">I", data, pos)
            pos += 4
            return v

        if u32() != 512:
            raise RasterError("expected header size indicator of 512")
        if pos + 512 > len(data):
            raise RasterError("truncated header")
        fields = struct.unpack_from(_HEADER_FMT, data, pos)
        pos += 512
        h1 = list(fields[:_H1])
        h2 = list(fields[_H1:_H1 + _H2])
        h3 = list(fields[_H1 + _H2:_H1 + _H2 + _H3])
        h4 = fields[_H1 + _H2 + _H3]
        h5 = list(fields[_H1 + _H2 + _H3 + 1:])
        if u32() != 512:
            raise RasterError("expected header size indicator of 512")
        block = u32()
        dtype_code, bpp = h1[11], h1[12]
        key = (dtype_code, bpp)
        if dtype_code not in (0, 1, 2):
            raise RasterError(f"unsupported NIMROD data type {dtype_code}")
        if key not in _DTYPES:
            raise RasterError(f"unsupported bytes per datum {bpp} for data type {dtype_code}")
        nrows, ncols = h1[15], h1[16]
        if nrows <= 0 or ncols <= 0:
            raise RasterError(f"bad grid size {ncols} x {nrows}")
        n = nrows * ncols
        size = n * bpp
        if pos + size > len(data):
            raise RasterError(f"could not read {size} bytes of data at offset {pos}")
        raw = np.frombuffer(data, dtype=_DTYPES[key], count=n, offset=pos).astype(np.float64)
        pos += size
        if u32() != block:
            raise RasterError(f"expected block size indicator matching {block}")
        self.nodata = float(np.float32(h2[6])) if dtype_code == 0 else float(h1[24])
        if h1[23] != 0:
            names = {1: "bottom-left", 2: "top-right", 3: "bottom-right"}
            raise RasterError(f"{names.get(h1[23], 'unknown')} grid origin location is not supported")
        self.header = {"h1": h1, "h2": h2, "h3": h3, "h4": h4, "h5": h5}
        self.scale, self.offset = float(np.float32(h2[7])), float(np.float32(h2[8]))
        f32 = [float(np.float32(v)) for v in h2]   # header reals, widened as the reader does
        dx, dy = f32[5], f32[3]
        llc_x = f32[4] - 0.5 * dx
        llc_y = f32[2] + (0.5 - float(nrows)) * dy
        urc_y = f32[2] + 0.5 * dy
        grid = raw.reshape(nrows, ncols)                           # north row first
        if bbox is not None:
            def px(v, lim):
                i = int(np.floor(v)) if np.isfinite(v) else 0
                return min(max(i, 0), lim - 1)
            c0 = px((bbox[0] - llc_x) / dx, ncols)
            r0 = px((urc_y - bbox[3]) / dy, nrows)
            c1 = px((bbox[2] - llc_x) / dx, ncols)
            r1 = px((urc_y - bbox[1]) / dy, nrows)
        else:
            c0, r0, c1, r1 = 0, 0, ncols - 1, nrows - 1
        self.ncols, self.nrows = c1 - c0 + 1, r1 - r0 + 1
        # lower-left corner of the kept area (NIMRODRasterFormat::llc, NIMROD.hpp:60-66)
        self.x0 = llc_x + c0 * dx
        self.y0 = llc_y + (nrows - r1 - 1) * dy
        self.dx, self.dy = dx, dy
        self.values = np.ascontiguousarray(grid[r0:r1 + 1, c0:c1 + 1][::-1])   # row 0 = south

    def cell_index(self, x, y):
        """Raster cell containing each location (row-major, row 0 south), or -1 outside
        (Cartesian2DMesh::get_coordinate and get_nearest_object_index for an unrotated mesh)."""
        x = np.asarray(x, np.float64)
        y = np.asarray(y, np.float64)
        cx = (x - self.x0) * (1.0 / self.dx)
        cy = (y - self.y0) * (1.0 / self.dy)
        inside = (cx >= 0.0) & (cx < self.ncols) & (cy >= 0.0) & (cy < self.nrows)
        ix = np.where(inside, cx, 0.0).astype(np.int64)
        iy = np.where(inside, cy, 0.0).astype(np.int64)
        return np.where(inside, iy * self.ncols + ix, -1)

    def map_to_mesh(self, nx, ny, dx, dy, origin=(0.0, 0.0), cells=None, field=None):
        """The raster on a solver mesh (MapFieldOperator): each selected cell (all when `cells`
        is None) takes the value of the raster cell containing its centre; others keep
        `field`'s value (zeros when `field` is None). Returns an (ny, nx) FP64 array."""
        out = np.zeros(nx * ny) if field is None else np.array(field, np.float64).reshape(-1)
        idx = np.arange(nx * ny) if cells is None else np.asarray(cells, np.int64)
        xi = (idx % nx).astype(np.float64) + 0.5
        yi = (idx // nx).astype(np.float64) + 0.5
        x = origin[0] + xi * dx + yi * 0.0           # Cartesian2DMesh::get_location
        y = origin[1] + xi * 0.0 + yi * dy
        j = self.cell_index(x, y)
        ok = j >= 0
        out[idx[ok]] = self.values.reshape(-1)[j[ok]]
        return out.reshape(ny, nx)


def nimrod_bytes(values, x_first, y_first, dx, dy, dtype="f4", nodata=-1.0, h1=None, h2=None, h4=b""):
    """A NIMROD file image: `values` (nrows x ncols, north row first) with the first pixel
    centre at (x_first, y_first) and intervals dx, dy; `dtype` one of f4, i2, i4, i1. Header
    entries not given are the format's missing values (-32767 and -32767.0)."""
    values = np.asarray(values)
    nrows, ncols = values.shape
    code, bpp = {"f4": (0, 4), "i2": (1, 2), "i4": (1, 4), "i1": (2, 1)}[dtype]
    a = [-32767] * _H1
    a[11], a[12], a[14], a[15], a[16], a[23] = code, bpp, 0, nrows, ncols, 0
    if code != 0:
        a[24] = int(nodata)
    for k, v in (h1 or {}).items():
        a[k] = v
    b = [-32767.0] * _H2
    b[2], b[3], b[4], b[5] = y_first, dy, x_first, dx
    if code == 0:
        b[6] = nodata
    b[7], b[8] = 1.0, 0.0
    for k, v in (h2 or {}).items():
        b[k] = v
    header = struct.pack(_HEADER_FMT, *a, *b, *([-32767.0] * _H3), h4.ljust(_H4, b" ")[:_H4], *([-32767] * _H5))
    body = np.ascontiguousarray(values, dtype=_DTYPES[(code, bpp)]).tobytes()
    return (struct.pack(">I", 512) + header + struct.pack(">I", 512) + struct.pack(">I", len(body)) + body +
            struct.pack(">I", len(body)))


__all__ = ["RasterError", "NimrodRaster", "nimrod_bytes"]
