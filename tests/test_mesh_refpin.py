"""Cell lookups against the reference's own mesh (CPU; needs the reference source tree).

The raster mapping (mfcm_b200/raster.py) and the depth-point measure (mfcm_b200/outputs.py)
find the cell that contains a location, and the outputs write cell centres. The reference does
both in Cartesian2DMesh (get_nearest_object_index<Cell> and get_object_location<Cell>,
src/Mesh/Cartesian2DMesh.hpp:139-188), which oracle/ref_pin compiles; the package must give the
same cell and the same centre, bit for bit, on cell edges and just beside them too.
"""
import numpy as np
import pytest

from mfcm_b200 import outputs
from mfcm_b200.raster import NimrodRaster
from oracle.ref_pin import refpin

pytestmark = pytest.mark.skipif(not refpin.available(), reason="reference source tree not present")

MESHES = [(4, 3, 0.1, 0.3, (1.0, 2.0)), (7, 5, 2.0, 2.0, (0.0, 0.0)), (9, 2, 0.37, 5.3, (-1234.5, 77.25)),
          (1, 6, 1000.0, 250.0, (400000.0, 100000.0)), (5, 5, 0.7, 0.7, (0.3, -0.9))]


def _locations(nx, ny, dx, dy, origin, rng):
    ox, oy = origin
    xs = [ox + k * dx for k in range(nx + 1)] + [ox + (k + 0.5) * dx for k in range(nx)]
    ys = [oy + k * dy for k in range(ny + 1)] + [oy + (k + 0.5) * dy for k in range(ny)]
    xs = xs + [np.nextafter(x, -np.inf) for x in xs] + [np.nextafter(x, np.inf) for x in xs]
    ys = ys + [np.nextafter(y, -np.inf) for y in ys] + [np.nextafter(y, np.inf) for y in ys]
    gx, gy = np.meshgrid(np.array(xs), np.array(ys))
    rx = rng.uniform(ox - 2 * dx, ox + (nx + 2) * dx, 200)
    ry = rng.uniform(oy - 2 * dy, oy + (ny + 2) * dy, 200)
    return np.concatenate([gx.ravel(), rx]), np.concatenate([gy.ravel(), ry])


@pytest.mark.parametrize("mesh", MESHES)
def test_cell_lookup_and_centres_match_reference(mesh):
    nx, ny, dx, dy, origin = mesh
    rng = np.random.default_rng(nx * 13 + ny)
    x, y = _locations(nx, ny, dx, dy, origin, rng)
    ref, (cx, cy) = refpin.nearest_cells(nx, ny, dx, dy, origin, x, y)
    assert np.any(ref == nx * ny) and np.any(ref < nx * ny)
    # cell centres, as the outputs write them
    ox_, oy_ = outputs.cell_locations(nx, ny, dx, dy, *origin)
    assert np.array_equal(ox_.view(np.int64), cx.view(np.int64))
    assert np.array_equal(oy_.view(np.int64), cy.view(np.int64))
    # the raster mapping's lookup (a raster of the mesh's geometry)
    r = NimrodRaster.__new__(NimrodRaster)
    r.x0, r.y0, r.dx, r.dy, r.ncols, r.nrows = origin[0], origin[1], dx, dy, nx, ny
    got = r.cell_index(x, y)
    assert np.array_equal(np.where(got < 0, nx * ny, got), ref)
    # the depth-point measure's cell (a location outside the mesh is refused)
    for xi, yi, ri in zip(x, y, ref):
        if ri == nx * ny:
            with pytest.raises(ValueError):
                outputs.DepthPointMeasure((xi, yi), nx, ny, dx, dy, origin)
        else:
            assert outputs.DepthPointMeasure((xi, yi), nx, ny, dx, dy, origin).index == ri, (xi, yi)
