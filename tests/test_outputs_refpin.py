"""The output files (mfcm_b200/outputs.py) against the reference's own formatters (CPU; needs
the reference source tree).

oracle/ref_pin/build.py compiles the reference's CSVOutput and RawBinaryOutput
(src/Output/OutputFormat.hpp) with FieldOutputFunction and TimeSeriesOutputFunction
(src/Output/OutputFunction.hpp) over its own mesh and field classes. The same cell fields and
measure points are written by both, and the files must be equal byte for byte: names quoted
as std::quoted does, values as std::to_string does (a NaN with its sign bit set included),
cell-centre locations as an ostream writes a double, every delimiter, both value types.
Without the reference tree the tests skip.
"""
import numpy as np
import pytest

from mfcm_b200 import outputs
from oracle.ref_pin import refpin

pytestmark = pytest.mark.skipif(not refpin.available(), reason="reference source tree not present")

NAMES = ["h", "u", "stage", 'we"ird', "back\\slash", "with space", "depth m³/s", "ünïcode"]
DELIMITERS = [", ", ";", "\t", " | ", ","]


def _values(rng, n, dtype):
    v = rng.normal(0.0, 1.0, n) * 10.0 ** rng.integers(-9, 9, n)
    special = [np.nan, -np.nan, np.inf, -np.inf, -0.0, 0.0, 5e-7, 4.9999995e-7, 1e300, -2.5e-310, 123456.789]
    k = rng.choice(n, min(n, len(special)), replace=False)
    v[k] = special[:len(k)]
    # an invalid operation gives x86's default NaN, whose sign bit is set
    with np.errstate(invalid="ignore"):
        if n > len(special):
            v[rng.integers(0, n)] = np.float64(np.inf) - np.float64(np.inf)
    with np.errstate(over="ignore"):  # 1e300 becomes inf in FP32, as in the solver's value type
        return v.astype(dtype)


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("seed", range(6))
def test_field_csv_matches_reference(tmp_path, prec, seed):
    rng = np.random.default_rng(seed)
    dtype = np.float64 if prec == "f64" else np.float32
    nx, ny = int(rng.integers(1, 9)), int(rng.integers(1, 7))
    dx, dy = float(rng.choice([0.5, 2.0, 3.7, 1000.0])), float(rng.choice([0.25, 2.0, 5.3]))
    origin = (float(rng.uniform(-1e6, 1e6)), float(rng.uniform(-1e3, 1e3))) if seed % 2 else (0.0, 0.0)
    k = int(rng.integers(1, 5))
    names = list(rng.choice(NAMES, k, replace=False))
    cols = [_values(rng, nx * ny, dtype) for _ in range(k)]
    delim = DELIMITERS[seed % len(DELIMITERS)]
    ref_path = tmp_path / "ref.csv"
    refpin.write_fields(str(ref_path), nx, ny, dx, dy, origin, names, cols, delimiter=delim, precision=prec)
    ours_path = tmp_path / "ours.csv"
    loc = outputs.cell_locations(nx, ny, dx, dy, *origin)
    outputs.write_csv(str(ours_path), names, cols, loc, delim)
    assert ours_path.read_bytes() == ref_path.read_bytes()


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_raw_binary_matches_reference(tmp_path, prec):
    rng = np.random.default_rng(11)
    dtype = np.float64 if prec == "f64" else np.float32
    nx, ny = 7, 5
    cols = [_values(rng, nx * ny, dtype) for _ in range(3)]
    ref_path = tmp_path / "ref.bin"
    refpin.write_fields(str(ref_path), nx, ny, 2.0, 2.0, (0.0, 0.0), ["h", "u", "v"], cols, binary=True,
                        precision=prec)
    assert outputs.raw_binary_bytes(cols, dtype) == ref_path.read_bytes()
    back, n = outputs.read_raw_binary(ref_path.read_bytes())
    assert n == len(ref_path.read_bytes())
    np.testing.assert_array_equal(back.view(np.uint8), np.stack(cols, axis=1).view(np.uint8))


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_measure_csv_matches_reference(tmp_path, prec):
    """A depth-point measure's file, times and depths in the solver's value type."""
    rng = np.random.default_rng(5)
    dtype = np.float64 if prec == "f64" else np.float32
    times = np.cumsum(rng.uniform(0.1, 900.0, 12))
    depths = _values(rng, 12, dtype)
    ref_path = tmp_path / "ref.csv"
    refpin.write_series(str(ref_path), times, depths, "gauge \"A\"", precision=prec)
    m = outputs.DepthPointMeasure((1.0, 1.0), 2, 2, 2.0, 2.0, name="gauge \"A\"", value_type=dtype)
    m.points = [(float(t), float(d)) for t, d in zip(times, depths)]
    ours_path = tmp_path / "ours.csv"
    m.write(str(ours_path))
    assert ours_path.read_bytes() == ref_path.read_bytes()
