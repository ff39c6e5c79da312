"""Outputs, measures and checkpoints of a solve, in the reference's file formats.

- Timed multi-field CSV files (MultiFieldOutputFile, src/Output/OutputFile.hpp:159-224): one file
  `<name>_<std::to_string(t)>.csv` whenever t reaches start + every * n. Each file has a header
  `X, Y, "f1", "f2", ` and one row per cell `x, y, v1, v2, `, the delimiter ", " ending every
  entry (CSVOutput, src/Output/OutputFormat.hpp:78-122). Names are quoted as std::quoted
  quotes them. Coordinates are written as a C++ ostream writes a double (precision 6, %g);
  values as std::to_string does (%f, OutputFunction.hpp:88-92), a NaN with its sign bit set
  as glibc's "-nan".
- Raw binary (RawBinaryOutput, OutputFormat.hpp:47-76): three 64-bit unsigned integers
  (rows, columns, bytes per value), then the values row by row in the value type.
- Measures (src/SaintVenant/Measure.hpp:57-177): the volume of the wetted domain and the depth
  at the cell nearest a location, one point per update, written as a time series CSV with
  columns "ID" (the time) and the measure's name.
- Checkpoints: the state h, u, v (with the infiltration capacity when that term is active,
  and the FP32 solvers' depth-update compensation) as one raw binary block in the solver's
  value type, followed by a JSON trailer with the
  timestep, the running counters and tallies and the mesh. Restoring one into a solver of
  the same shape and precision continues the solve bit for bit. The reference has no restart.

Field names follow the reference: "h", "u", "v" (State.hpp:139-149), "stage" (z_bed + h,
Solver.hpp:90-98; formed here in FP64 from the host copies), "z_bed" (Constants.hpp:39),
"fx" and "fy" (energy-loss coefficients, EnergyLossSourceTerm.hpp:236-243; also under their
input-field names "fdx" and "fdy"), and "IR" and "IC" (infiltration rate and capacity).
"""
import json
import math
import os
import struct

import numpy as np

from . import FIELD

_NAMES = {"h": "H", "u": "U", "v": "V", "z_bed": "Z", "IR": "INFIL_RATE", "IC": "INFIL_CAP",
          "fx": "ELOSS_FX", "fy": "ELOSS_FY", "fdx": "ELOSS_FX", "fdy": "ELOSS_FY", "h_comp": "H_COMP"}


def _signed_nan(x, text):
    """glibc's printf writes a NaN with its sign bit set as "-nan"."""
    if x != x and math.copysign(1.0, x) < 0.0:
        return "-" + text
    return text


def fmt_value(x):
    """std::to_string(double): printf %f."""
    return _signed_nan(x, "%f" % x)


def fmt_coord(x):
    """operator<<(std::ostream&, double) with the default precision 6: printf %g."""
    return _signed_nan(x, "%g" % x)


def quoted(name):
    """std::quoted(name) on output: the name in double quotes, with every double quote and
    backslash preceded by a backslash; everything else, non-ASCII text included, as is."""
    return '"' + name.replace("\\", "\\\\").replace('"', '\\"') + '"'


def cell_locations(nx, ny, dx, dy, origin_x=0.0, origin_y=0.0):
    """Cell centres (Cartesian2DMesh::get_object_location<Cell>, Cartesian2DMesh.hpp:139-146,
    unrotated mesh): x = ox + (i % nx + 0.5) dx, y = oy + (i / nx + 0.5) dy."""
    i = np.arange(nx * ny)
    xi = (i % nx).astype(np.float64) + 0.5
    yi = (i // nx).astype(np.float64) + 0.5
    return origin_x + xi * dx + yi * 0.0, origin_y + xi * 0.0 + yi * dy


def csv_text(names, columns, locations=None, delimiter=", "):
    """CSVOutput::output as text. `columns` are equal-length 1-D arrays; `locations` an
    (x, y) pair of arrays or None."""
    q = [quoted(n) for n in names]
    head = (["X", "Y"] if locations is not None else []) + q
    lines = ["".join(h + delimiter for h in head)]
    cols = [np.asarray(c).ravel() for c in columns]
    n = len(cols[0]) if cols else 0
    for r in range(n):
        parts = []
        if locations is not None:
            parts += [fmt_coord(float(locations[0][r])), fmt_coord(float(locations[1][r]))]
        parts += [fmt_value(float(c[r])) for c in cols]
        lines.append("".join(p + delimiter for p in parts))
    return "\n".join(lines) + "\n"


def write_csv(path, names, columns, locations=None, delimiter=", "):
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    with open(path, "w", encoding="utf-8", newline="\n") as f:
        f.write(csv_text(names, columns, locations, delimiter))


def raw_binary_bytes(columns, dtype=np.float64):
    """RawBinaryOutput::output as bytes: nrows, ncols, value size, then row-major values."""
    cols = [np.asarray(c, dtype=dtype).ravel() for c in columns]
    nrows = len(cols[0]) if cols else 0
    body = np.stack(cols, axis=1) if cols else np.zeros((0, 0), dtype=dtype)
    return struct.pack("<QQQ", nrows, len(cols), np.dtype(dtype).itemsize) + body.astype(dtype).tobytes()


def read_raw_binary(data):
    """Inverse of raw_binary_bytes: returns an (nrows, ncols) array and the number of bytes read."""
    nrows, ncols, size = struct.unpack_from("<QQQ", data, 0)
    dtype = {4: np.float32, 8: np.float64}[size]
    n = nrows * ncols * size
    arr = np.frombuffer(data, dtype=dtype, count=nrows * ncols, offset=24).reshape(nrows, ncols)
    return arr, 24 + n


def solver_field(solver, name):
    """A named output field of a solver (host copy, FP64)."""
    if name == "stage":
        return solver.get_field("Z") + solver.get_field("H")
    if name not in _NAMES:
        raise KeyError(f"no output field {name!r}")
    return solver.get_field(_NAMES[name])


class MultiFieldOutput:
    """TimedOutputFile + MultiFieldOutputFile (OutputFile.hpp:121-224): named cell fields to
    `<base>_<std::to_string(t)>.csv` every `every` seconds from `start`."""

    def __init__(self, base, fields, every, start=0.0, origin=(0.0, 0.0), delimiter=", "):
        self.base = base
        self.delimiter = delimiter
        self.fields = list(fields)
        self.every = float(every)
        self.start = float(start)
        self.origin = origin
        self.output_no = 0
        self.written = []

    def timed_output(self, t, solver):
        if not (t >= self.start + self.every * self.output_no):
            return None
        path = f"{self.base}_{fmt_value(t)}.csv"
        loc = cell_locations(solver.nx, solver.ny, solver.dx, solver.dy, *self.origin)
        write_csv(path, self.fields, [solver_field(solver, f) for f in self.fields], loc, self.delimiter)
        self.output_no += 1
        self.written.append(path)
        return path


class VolumeMeasure:
    """SaintVenantVolumeMeasure (Measure.hpp:137-177): sum of h times the cell area, per update."""

    def __init__(self, name="volume"):
        self.name = name
        self.points = []

    def update(self, t, solver):
        self.points.append((float(t), float(solver.stats()["volume"])))

    def write(self, path):
        write_csv(path, ["ID", self.name], [[p[0] for p in self.points], [p[1] for p in self.points]])


class DepthPointMeasure:
    """SaintVenantHPointMeasure (Measure.hpp:57-135): the depth of the cell nearest `location`
    (Cartesian2DMesh::get_nearest_object_index<Cell>, Cartesian2DMesh.hpp:179-188); a location
    outside the mesh is an error (the reference would read past the field). `value_type` is the
    solver's: the reference's time series output writes the times in it too
    (TimeSeriesOutputFunction::at, Output/OutputFunction.hpp:373-383)."""

    def __init__(self, location, nx, ny, dx, dy, origin=(0.0, 0.0), name="h_point", value_type=np.float64):
        # Cartesian2DMesh::get_coordinate (Cartesian2DMesh.hpp:112-121) on an unrotated mesh:
        # the offset times the stored reciprocal of the cell size, which rounds differently from
        # a division on cell edges
        cx = (location[0] - origin[0]) * (1.0 / dx)
        cy = (location[1] - origin[1]) * (1.0 / dy)
        if not (0.0 <= cx < nx and 0.0 <= cy < ny):
            raise ValueError(f"location {location} is outside the mesh")
        self.index = int(math.floor(cy)) * nx + int(math.floor(cx))
        self.name = name
        self.value_type = value_type
        self.points = []

    def update(self, t, solver):
        self.points.append((float(t), float(solver.get_field("H").ravel()[self.index])))

    def write(self, path):
        vt = self.value_type
        write_csv(path, ["ID", self.name], [np.array([p[0] for p in self.points], dtype=vt),
                                             np.array([p[1] for p in self.points], dtype=vt)])


_CKPT_MAGIC = b"SVCKPT01"


def save_checkpoint(solver, path, t=None, infiltration=False):
    """Write the state (h, u, v, and the infiltration capacity if `infiltration`) as a raw
    binary block in the solver's value type, then a JSON trailer: dt, the running counters and
    tallies, the mesh, the precision and the simulated time `t`."""
    dtype = np.float64 if getattr(solver, "precision", "f64") == "f64" else np.float32
    # FP32 solvers carry a compensation of the depth update: part of the state
    comp = getattr(solver, "depth_compensation", False)
    names = ["h", "u", "v"] + (["IC"] if infiltration else []) + (["h_comp"] if comp else [])
    block = raw_binary_bytes([solver_field(solver, n) for n in names], dtype)
    meta = {"fields": names, "dt": solver.get_dt(), "stats": solver.stats(), "t": t,
            "nx": solver.nx, "ny": solver.ny, "dx": solver.dx, "dy": solver.dy,
            "precision": getattr(solver, "precision", "f64")}
    trailer = json.dumps(meta).encode()
    with open(path, "wb") as f:
        f.write(block + _CKPT_MAGIC + struct.pack("<Q", len(trailer)) + trailer)


def load_checkpoint(solver, path):
    """Restore a checkpoint into a solver of the same mesh and precision (the bed, roughness,
    forcing and other inputs are set by the caller as for any solve). Returns the trailer."""
    data = open(path, "rb").read()
    arr, n = read_raw_binary(data)
    if data[n:n + len(_CKPT_MAGIC)] != _CKPT_MAGIC:
        raise ValueError("not a checkpoint file")
    (m,) = struct.unpack_from("<Q", data, n + len(_CKPT_MAGIC))
    meta = json.loads(data[n + len(_CKPT_MAGIC) + 8:n + len(_CKPT_MAGIC) + 8 + m].decode())
    if (meta["nx"], meta["ny"]) != (solver.nx, solver.ny):
        raise ValueError("checkpoint mesh does not match the solver")
    if meta["precision"] != getattr(solver, "precision", "f64"):
        raise ValueError("checkpoint precision does not match the solver")
    shape = (solver.ny, solver.nx)
    for k, name in enumerate(meta["fields"]):  # the depth first: setting it clears the compensation
        solver.set_field(_NAMES[name], arr[:, k].astype(np.float64).reshape(shape))
    solver.set_dt(meta["dt"])
    solver.set_stats(meta["stats"])
    return meta


__all__ = ["fmt_value", "fmt_coord", "quoted", "cell_locations", "csv_text", "write_csv", "raw_binary_bytes",
           "read_raw_binary", "solver_field", "MultiFieldOutput", "VolumeMeasure", "DepthPointMeasure",
           "save_checkpoint", "load_checkpoint", "FIELD"]
