"""NIMROD raster input (mfcm_b200/raster.py): the file layout, value types, no-data values,
cropping and orientation, and the mapping onto a solver mesh, including through a
configuration deck. The reference ships no NIMROD files; these files are written by
`nimrod_bytes`, which restates the layout the reference's reader expects."""
import struct

import numpy as np
import pytest

from mfcm_b200 import config
from mfcm_b200.raster import NimrodRaster, RasterError, nimrod_bytes


def _grid(nrows, ncols, seed=0):
    return np.random.default_rng(seed).uniform(0.0, 50.0, (nrows, ncols)).astype(np.float32)


def test_layout_orientation_and_geometry():
    g = _grid(6, 9)
    r = NimrodRaster.from_bytes(nimrod_bytes(g, x_first=1000.0, y_first=2250.0, dx=100.0, dy=50.0, nodata=-1.0))
    assert (r.ncols, r.nrows, r.dx, r.dy) == (9, 6, 100.0, 50.0)
    assert r.x0 == 950.0                      # first pixel centre minus half a pixel
    assert r.y0 == 2250.0 + (0.5 - 6) * 50.0  # the southern edge
    assert np.array_equal(r.values, g[::-1].astype(np.float64))   # row 0 is the southern row
    assert r.nodata == -1.0 and r.header["h1"][15] == 6 and r.header["h1"][16] == 9


@pytest.mark.parametrize("dtype,nodata", [("f4", -1.0), ("i2", -1), ("i4", -9999), ("i1", -128)])
def test_value_types(dtype, nodata):
    g = (np.arange(12).reshape(3, 4) * 3 - 5).astype(np.float64)
    g[1, 2] = nodata
    r = NimrodRaster.from_bytes(nimrod_bytes(g, 0.5, 2.5, 1.0, 1.0, dtype=dtype, nodata=nodata))
    assert np.array_equal(r.values, g[::-1])          # values as stored, no-data kept
    assert r.nodata == float(nodata)


def test_scale_and_offset_are_reported_not_applied():
    g = np.array([[32, 64]], dtype=np.int16)
    r = NimrodRaster.from_bytes(nimrod_bytes(g, 0.5, 0.5, 1.0, 1.0, dtype="i2", h2={7: 0.03125, 8: 1.0}))
    assert r.scale == 0.03125 and r.offset == 1.0
    assert list(r.values.ravel()) == [32.0, 64.0]


def test_malformed_files():
    good = nimrod_bytes(_grid(2, 3), 0.5, 1.5, 1.0, 1.0)
    bad = [
        struct.pack(">I", 500) + good[4:],                          # header length
        good[:-10],                                                  # truncated data
        good[:-4] + struct.pack(">I", 7),                            # trailing block length
        nimrod_bytes(_grid(2, 3), 0.5, 1.5, 1.0, 1.0, h1={12: 2}),   # float with 2 bytes
        nimrod_bytes(_grid(2, 3), 0.5, 1.5, 1.0, 1.0, h1={11: 7}),   # unknown type
        nimrod_bytes(_grid(2, 3), 0.5, 1.5, 1.0, 1.0, h1={23: 1}),   # bottom-left origin
        nimrod_bytes(_grid(2, 3), 0.5, 1.5, 1.0, 1.0, h1={15: -2}),  # negative row count
        nimrod_bytes(_grid(2, 3), 0.5, 1.5, 1.0, 1.0, h1={16: 0}),   # no columns
    ]
    for b in bad:
        with pytest.raises(RasterError):
            NimrodRaster.from_bytes(b)
    for box in ([0, 0, 0, 1], [0, 1, 1, 1], [0, 1, 2]):
        with pytest.raises(RasterError):
            NimrodRaster.from_bytes(good, bbox=box)


def test_bounding_box_crop():
    g = _grid(10, 12, seed=3)
    data = nimrod_bytes(g, x_first=5.0, y_first=95.0, dx=10.0, dy=10.0)   # covers x 0..120, y 0..100
    r = NimrodRaster.from_bytes(data, bbox=[21.0, 33.0, 58.0, 71.0])
    # columns floor((21-0)/10)=2 .. floor((58-0)/10)=5; rows from the north edge y=100:
    # floor((100-71)/10)=2 .. floor((100-33)/10)=6
    assert (r.ncols, r.nrows) == (4, 5)
    assert np.array_equal(r.values, g[2:7, 2:6][::-1].astype(np.float64))
    assert (r.x0, r.y0) == (20.0, 30.0)       # the crop's own lower-left corner
    # a box larger than the file keeps all of it
    r2 = NimrodRaster.from_bytes(data, bbox=[-50.0, -50.0, 500.0, 500.0])
    assert (r2.ncols, r2.nrows, r2.x0, r2.y0) == (12, 10, 0.0, 0.0)


def test_map_onto_a_finer_offset_mesh():
    g = np.arange(12, dtype=np.float32).reshape(3, 4)       # 4 x 3 pixels of 10 m from (0, 0)
    r = NimrodRaster.from_bytes(nimrod_bytes(g, 5.0, 25.0, 10.0, 10.0))
    nx, ny, d = 10, 8, 5.0
    out = r.map_to_mesh(nx, ny, d, d, origin=(-7.5, 2.5), field=np.full((ny, nx), -3.0))
    for j in range(ny):
        for i in range(nx):
            x, y = -7.5 + (i + 0.5) * d, 2.5 + (j + 0.5) * d
            if 0 <= x < 40 and 0 <= y < 30:
                expect = g[::-1][int(y // 10), int(x // 10)]
            else:
                expect = -3.0                                # outside: previous value kept
            assert out[j, i] == expect, (i, j)
    # a selection writes each selected cell at its own index
    sel = np.array([5, 17, 63])
    out2 = r.map_to_mesh(nx, ny, d, d, origin=(-7.5, 2.5), cells=sel, field=np.full((ny, nx), -3.0))
    changed = np.flatnonzero(out2.ravel() != -3.0)
    assert list(changed) == [5, 17] and np.array_equal(out2.ravel()[sel], out.ravel()[sel])  # 63 is outside


def test_raster_fields_in_a_deck(tmp_path):
    g = np.linspace(1.0, 2.0, 48, dtype=np.float32).reshape(6, 8)
    (tmp_path / "dem.nim").write_bytes(nimrod_bytes(g, x_first=1.0, y_first=11.0, dx=2.0, dy=2.0))
    deck = tmp_path / "run.mf"
    deck.write_text("""
mesh
{
  cell count == 8 6
  cell size == 2 2
}
scheme == runge-kutta
{
  end time == 1
}
raster field == dem
{
  source == NIMROD
  filename == dem.nim
}
raster field == part
{
  source == nimrod
  filename == dem.nim
  bbox == 4 4 11 9
}
field == z_bed
{
  set == raster
  {
    name == dem
  }
  multiply == composite
  {
    model == constant
    {
      value == 3
      cells == id list
      {
        ids == 0 1
      }
    }
  }
}
field == n
{
  set == 0.5
  add == raster
  {
    name == part
  }
}
""")
    m = config.load(str(deck))
    z = m.field("z_bed", 0.0)
    expect = g[::-1].astype(np.float64)
    expect.ravel()[:2] *= 3.0
    assert np.array_equal(z, expect)
    part = NimrodRaster(str(tmp_path / "dem.nim"), bbox=[4, 4, 11, 9])
    n = m.field("n", 0.0)
    assert np.array_equal(n, 0.5 + part.map_to_mesh(8, 6, 2.0, 2.0))
    deck.write_text(deck.read_text().replace("source == NIMROD", "source == gdal"))
    with pytest.raises(config.ConfigError, match="GDAL"):
        config.load(str(deck)).field("z_bed", 0.0)
