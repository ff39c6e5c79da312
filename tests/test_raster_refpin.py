"""The NIMROD reader (mfcm_b200/raster.py) against the reference's own reader (CPU; needs the
reference source tree).

oracle/ref_pin/build.py compiles the reference's NIMRODRasterFormat (src/Raster/RasterFormats/
NIMROD.cpp:313-566) unchanged into oracle/_ref/libsv_refpin_nimrod.so; oracle/ref_pin/refpin.py
runs it on a file and returns everything it read. Both readers get the same files, written by
`nimrod_bytes`, and must agree bit for bit on the header arrays, the grid, the no-data value,
the geotransform and, for bounding boxes inside the grid, the crop and its corner. Where the
reference's crop is wrong (the bugs the package fixes) the tests show the reference's result
beside the package's. Malformed files must fail in both. Without the reference tree the tests
skip.
"""
import struct

import numpy as np
import pytest

from mfcm_b200.raster import NimrodRaster, RasterError, nimrod_bytes
from oracle.ref_pin import refpin

pytestmark = pytest.mark.skipif(not refpin.available(), reason="reference source tree not present")

TYPES = {"f4": (np.float32, -1.0), "i2": (np.int16, -32767), "i4": (np.int32, -1), "i1": (np.int8, -128)}


def _values(dtype, nrows, ncols, rng):
    t, nodata = TYPES[dtype]
    if dtype == "f4":
        v = rng.lognormal(0.0, 1.5, (nrows, ncols)).astype(np.float32)
    else:
        info = np.iinfo(t)
        v = rng.integers(info.min + 1, info.max, (nrows, ncols), endpoint=True).astype(t)
    v[rng.uniform(size=v.shape) < 0.1] = nodata
    return v, nodata


def _geometry(rng):
    """First pixel centre and intervals, as the header's float32 values."""
    dx = float(np.float32(rng.choice([1000.0, 250.0, 5.0, 0.37, 2.5])))
    dy = float(np.float32(dx * rng.choice([1.0, 1.0, 0.5, 2.0])))
    x0 = float(np.float32(rng.uniform(-5e5, 7e5)))
    y0 = float(np.float32(rng.uniform(-1e5, 1.2e6)))
    return x0, y0, dx, dy


def _write(tmp_path, name, data):
    p = tmp_path / name
    p.write_bytes(data)
    return str(p)


def _same(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    return a.shape == b.shape and np.array_equal(a.view(np.int64), b.view(np.int64))


@pytest.mark.parametrize("dtype", list(TYPES))
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_header_grid_and_geometry(tmp_path, dtype, seed):
    rng = np.random.default_rng(100 * seed + len(dtype))
    nrows, ncols = int(rng.integers(1, 70)), int(rng.integers(1, 90))
    v, nodata = _values(dtype, nrows, ncols, rng)
    x0, y0, dx, dy = _geometry(rng)
    h1 = {0: 2024, 1: 6, 13: int(rng.integers(0, 100))}
    h2 = {7: 0.03125, 8: -2.0, 20: float(np.float32(rng.normal()))}
    path = _write(tmp_path, "g.dat", nimrod_bytes(v, x0, y0, dx, dy, dtype=dtype, nodata=nodata, h1=h1, h2=h2,
                                                  h4=b"rain rate mm/h"))
    ref = refpin.nimrod_read(path)
    ours = NimrodRaster(path)
    # header arrays as read
    assert ref["h1"] == ours.header["h1"]
    assert _same(ref["h2"], ours.header["h2"]) and _same(ref["h3"], ours.header["h3"])
    assert ref["h4"] == ours.header["h4"]
    assert ref["h5"] == ours.header["h5"]
    # the grid as stored (file order, north row first; the package keeps row 0 to the south)
    assert (ref["nypx"], ref["nxpx"]) == (nrows, ncols)
    assert _same(ref["buffer"], ours.values[::-1])
    assert _same(ref["buffer"], v.astype(np.float64))
    assert _same([ref["nodata"]], [ours.nodata])
    # geotransform: lower-left corner of the whole grid, pixel sizes
    assert _same(ref["geo"], [ours.x0, ours.dx, 0.0, ours.y0, 0.0, ours.dy])
    assert (ref["ncols"], ref["nrows"]) == (ours.ncols, ours.nrows)


@pytest.mark.parametrize("dtype", ["f4", "i2"])
def test_crops_inside_the_grid(tmp_path, dtype):
    rng = np.random.default_rng(7 + len(dtype))
    checked = 0
    for case in range(25):
        nrows, ncols = int(rng.integers(2, 60)), int(rng.integers(2, 60))
        v, nodata = _values(dtype, nrows, ncols, rng)
        x0, y0, dx, dy = _geometry(rng)
        path = _write(tmp_path, f"c{case}.dat", nimrod_bytes(v, x0, y0, dx, dy, dtype=dtype, nodata=nodata))
        llx, urx = x0 - 0.5 * dx, x0 + (ncols - 0.5) * dx
        lly, ury = y0 + (0.5 - nrows) * dy, y0 + 0.5 * dy
        # corners strictly inside the grid, some on pixel edges
        fx = np.sort(rng.uniform(0.001, 0.999, 2))
        fy = np.sort(rng.uniform(0.001, 0.999, 2))
        if case % 5 == 0:
            fx = np.array([1, ncols - 1]) / ncols
            fy = np.array([1, nrows - 1]) / nrows
        bbox = (llx + fx[0] * (urx - llx), lly + fy[0] * (ury - lly), llx + fx[1] * (urx - llx),
                lly + fy[1] * (ury - lly))
        if not (bbox[2] > bbox[0] and bbox[3] > bbox[1]):
            continue
        ref = refpin.nimrod_read(path, bbox)
        ours = NimrodRaster(path, bbox=bbox)
        assert (ref["ncols"], ref["nrows"]) == (ours.ncols, ours.nrows), (case, bbox)
        assert _same(ref["values"], ours.values[::-1]), case
        # the crop's lower-left corner: the reader's own llc(), which the package uses
        assert _same(ref["llc"], [ours.x0, ours.y0]), case
        checked += 1
    assert checked >= 20


def test_reference_crop_findings(tmp_path):
    """What the package fixes: without a bounding box the reference keeps no values; its mesh
    corner is the whole grid's, not the crop's; a box reaching below the grid clamps the
    lower-right row to row 0 (the northern row) instead of the last."""
    rng = np.random.default_rng(5)
    v, nodata = _values("f4", 12, 10, rng)
    x0, y0, dx, dy = 1000.0, 5000.0, 10.0, 10.0
    path = _write(tmp_path, "f.dat", nimrod_bytes(v, x0, y0, dx, dy, nodata=nodata))
    ref = refpin.nimrod_read(path)
    assert ref["values"].size == 0
    assert NimrodRaster(path).values.size == 12 * 10

    bbox = (1012.0, 4912.0, 1047.0, 4978.0)
    ref = refpin.nimrod_read(path, bbox)
    ours = NimrodRaster(path, bbox=bbox)
    assert _same(ref["values"], ours.values[::-1])
    assert ref["geo"][0] == 995.0 and ref["geo"][3] == 4885.0      # the whole grid's corner
    assert ref["llc"] == (ours.x0, ours.y0) == (1005.0, 4905.0)     # the crop's

    low = (1012.0, 4800.0, 1047.0, 5001.0)      # top in the first row, bottom 85 m below the grid
    ref = refpin.nimrod_read(path, low)
    ours = NimrodRaster(path, bbox=low)
    assert ref["lrc"][1] == 0 and ref["nrows"] == 1 and _same(ref["values"], v[0, 1:6])
    assert ours.nrows == 12 and _same(ours.values[::-1], v[:, 1:6])


def _corrupt(data, offset, fmt, value):
    b = bytearray(data)
    struct.pack_into(fmt, b, offset, value)
    return bytes(b)


def test_malformed_files_fail_in_both(tmp_path):
    v = np.arange(20, dtype=np.float32).reshape(4, 5)
    good = nimrod_bytes(v, 10.0, 20.0, 1.0, 1.0)
    data_at = 4 + 512 + 4 + 4
    cases = {
        "first record length": _corrupt(good, 0, ">I", 511),
        "second record length": _corrupt(good, 4 + 512, ">I", 500),
        "data type": nimrod_bytes(v, 10.0, 20.0, 1.0, 1.0, h1={11: 3}),
        "float bytes per datum": nimrod_bytes(v, 10.0, 20.0, 1.0, 1.0, h1={12: 2}),
        "integer bytes per datum": nimrod_bytes(v.astype(np.int16), 10.0, 20.0, 1.0, 1.0, dtype="i2", h1={12: 8}),
        "char bytes per datum": nimrod_bytes(v.astype(np.int8), 10.0, 20.0, 1.0, 1.0, dtype="i1", h1={12: 2}),
        "bottom-left origin": nimrod_bytes(v, 10.0, 20.0, 1.0, 1.0, h1={23: 1}),
        "top-right origin": nimrod_bytes(v, 10.0, 20.0, 1.0, 1.0, h1={23: 2}),
        "bottom-right origin": nimrod_bytes(v, 10.0, 20.0, 1.0, 1.0, h1={23: 3}),
        "unknown origin": nimrod_bytes(v, 10.0, 20.0, 1.0, 1.0, h1={23: 9}),
        "trailing record length": good[:-4] + struct.pack(">I", 79),
        "truncated data": good[:data_at + 30],
        "truncated header": good[:300],
        "missing trailer": good[:-4],
    }
    for name, data in cases.items():
        path = _write(tmp_path, "bad.dat", data)
        with pytest.raises(refpin.RefReaderError):
            refpin.nimrod_read(path)
        with pytest.raises(RasterError):
            NimrodRaster(path)
    path = _write(tmp_path, "ok.dat", good)
    for bbox in [(12.0, 15.0, 11.0, 19.0), (11.0, 19.0, 12.0, 15.0), (11.0, 15.0, 11.0, 19.0)]:
        with pytest.raises(refpin.RefReaderError):
            refpin.nimrod_read(path, bbox)
        with pytest.raises(RasterError):
            NimrodRaster(path, bbox=bbox)


def test_record_lengths_are_only_matched(tmp_path):
    """Neither reader checks the data record's length against the grid size, only that its
    leading and trailing copies agree."""
    v = np.arange(6, dtype=np.float32).reshape(2, 3)
    data = nimrod_bytes(v, 0.5, 1.5, 1.0, 1.0)
    at = 4 + 512 + 4
    data = _corrupt(data, at, ">I", 7)
    data = data[:-4] + struct.pack(">I", 7)
    path = _write(tmp_path, "len.dat", data)
    ref = refpin.nimrod_read(path)
    ours = NimrodRaster(path)
    assert _same(ref["buffer"], ours.values[::-1])
