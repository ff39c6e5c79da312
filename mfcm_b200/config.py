"""Reads the reference's `.mf` configuration decks and drives a solve from one.

The reader follows the reference's parser (src/Config/mf_parser/mf_parser_read.hpp:207-408):

- a line is `key words == data`: the key is the words before `==`, joined by single
  spaces, and the data is the rest of the line, or a quoted string with escapes and `\\`
  continuations;
- a line holding `{` opens the children of the last key, and `}` closes them;
- `!` starts a comment, and `#include "file"` reads another file, relative to this one;
- repeated keys are kept in order, as in a Boost property tree.

On top of the tree sit the parts of the schema that drive this solver:

- the mesh (Cartesian2DMesh.cpp:30-40);
- the scheme and its time parameters, with the time parser's units (hours by default) or
  calendar times in a `time format` (TimeParameters.cpp:23-38, TimeParser.cpp:20-134);
- fields built by `set` / `add` / `multiply` of constant, sloped, composite or NIMROD raster
  inputs within global, id-list or point (WKT) selections (FieldGenerator.cpp:26-178,
  MeshSelection.cpp:146-193, Raster.cpp:35-68; the raster reader is mfcm_b200/raster.py);
- time series, inline or CSV (TimeSeries.cpp:179-296);
- the source terms: Manning roughness, infiltration, energy loss, eddy viscosity
  (SourceTerm.cpp:32-50), the momentum terms in their configured order;
- the boundaries: discharge, head, stage, each a list of constant or time-series entries on
  cell selections (DischargeBoundarySourceTerm.hpp:114-146 and siblings);
- outputs (`output == name`, cell fields as timed CSV files) and depth-point measures
  (`measures { h-point == name }`), written by `Model.solve`.

GDAL rasters and vector files, geometries other than points in selections, and face or vertex
outputs are not read: a deck that uses them raises ConfigError naming the feature.
"""
import datetime
import math
import os
import re

import numpy as np

from .raster import NimrodRaster, RasterError
from .outputs import MultiFieldOutput, DepthPointMeasure, _NAMES as _OUTPUT_FIELDS
from . import (TimeSeries, Forcing, num_steps, RAIN_NONE, RAIN_UNIFORM, RAIN_FIELDS, HEAD_NONE, HEAD_FIELDS,
               STAGE_FIELDS)



_SPACE = " \t\n\v\f\r"   # isspace in the C locale


def rapidcsv_rows(data, sep=",", comment="#"):
    """rapidcsv 8.51's Document::ParseCsv (the reader the reference vendors in src/rapidcsv/)
    with the reference's settings: cells split at `sep` outside quotes, a quote opening a quoted
    cell only at the cell's first character, carriage returns dropped, cells trimmed of
    whitespace and then unquoted (outer quotes removed, doubled quotes halved), empty lines
    skipped (a line of blanks is a row of one empty cell), lines whose first cell starts with
    `comment` skipped except a last line without a line break, a UTF-8 byte-order mark
    ignored. Bytes map one to one onto the characters of the returned cells (latin-1)."""
    if data[:3] == b"\xef\xbb\xbf":
        data = data[3:]
    text = data.decode("latin-1")

    def finish(cell):
        cell = cell.strip(_SPACE)
        if len(cell) >= 2 and cell[0] == '"' and cell[-1] == '"':
            cell = cell[1:-1].replace('""', '"')
        return cell

    rows, row, cell, quoted = [], [], "", False
    for ch in text:
        if ch == '"':
            if cell == "" or cell[0] == '"':
                quoted = not quoted
            cell += ch
        elif ch == sep:
            if quoted:
                cell += ch
            else:
                row.append(finish(cell))
                cell = ""
        elif ch == "\r":
            pass
        elif ch == "\n":
            if not row and cell == "":
                continue
            row.append(finish(cell))
            if not (row[0] != "" and row[0][0] == comment):
                rows.append(row)
            row, cell, quoted = [], "", False
        else:
            cell += ch
    if cell != "" or row:
        row.append(finish(cell))
        rows.append(row)
    return rows


_STRTOD = re.compile(r"[ \t\n\v\f\r]*[+-]?(?:(?P<inf>inf(?:inity)?)|(?P<nan>nan(?:\([0-9A-Za-z_]*\))?)"
                     r"|(?P<hex>0x(?:[0-9a-f]+\.?[0-9a-f]*|\.[0-9a-f]+)(?:p[+-]?[0-9]+)?)"
                     r"|(?P<dec>(?:[0-9]+\.?[0-9]*|\.[0-9]+)(?:e[+-]?[0-9]+)?))", re.IGNORECASE)


def stod_or_nan(cell):
    """rapidcsv's default converter for double: std::stod, i.e. strtod in the C locale on the
    longest valid prefix (leading blanks, a sign, decimal or hexadecimal digits, inf, nan), and
    NaN where std::stod throws: no number at the start, or a result out of range (overflow to
    infinity, or underflow below the smallest normal double)."""
    m = _STRTOD.match(cell)
    if not m:
        return float("nan")
    text = m.group(0).strip(_SPACE)
    if m.group("inf") or m.group("nan"):
        return float(text.lower().split("(")[0])
    try:
        v = float.fromhex(text) if m.group("hex") else float(text)
    except OverflowError:
        return float("nan")
    if math.isinf(v):
        return float("nan")
    if v == 0.0:
        digits = re.sub(r"[eEpP].*$", "", text)
        digits = re.sub(r"^[+-]?(0[xX])?", "", digits)
        if re.search(r"[1-9a-fA-F]", digits):
            return float("nan")  # a non-zero number that underflowed to zero
    elif abs(v) < 2.2250738585072014e-308:
        return float("nan")  # a subnormal result
    return v

class ConfigError(ValueError):
    pass


# ------------------------------------------------------------------------------------ tree
class Node:
    """A property-tree node: a value and an ordered list of (key, child) pairs."""

    def __init__(self, value=""):
        self.value = value
        self.children = []

    def add(self, key):
        n = Node()
        self.children.append((key, n))
        return n

    def equal_range(self, key):
        return [n for k, n in self.children if k == key]

    def child(self, key):
        r = self.equal_range(key)
        return r[0] if r else None

    def get(self, path, default=None):
        """Value at a dotted path (ptree.get); `default` when absent, ConfigError if required."""
        n = self
        for part in path.split("."):
            n = n.child(part)
            if n is None:
                if default is None:
                    raise ConfigError(f"missing configuration key {path!r}")
                return default
        return n.value

    def __iter__(self):
        return iter(self.children)


_ESCAPES = {"0": "\0", "a": "\a", "b": "\b", "f": "\f", "n": "\n", "r": "\r", "t": "\t", "v": "\v",
            '"': '"', "'": "'", "\\": "\\"}


def _expand(s):
    out, i = [], 0
    while i < len(s):
        c = s[i]
        if c == "\\":
            i += 1
            if i >= len(s) or s[i] not in _ESCAPES:
                raise ConfigError("unknown escape sequence")
            out.append(_ESCAPES[s[i]])
        else:
            out.append(c)
        i += 1
    return "".join(out)


def _isspace(c):
    return ord(c) < 128 and c.isspace()


class _Line:
    def __init__(self, text):
        self.t = text
        self.i = 0

    def skip(self):
        while self.i < len(self.t) and _isspace(self.t[self.i]):
            self.i += 1

    def peek(self):
        return self.t[self.i] if self.i < len(self.t) else "\0"

    def word(self):
        self.skip()
        s = self.i
        while self.i < len(self.t) and not _isspace(self.t[self.i]) and self.t[self.i] != "!":
            self.i += 1
        return _expand(self.t[s:self.i])

    def rest(self):
        self.skip()
        s = self.i
        while self.i < len(self.t) and self.t[self.i] != "!":
            self.i += 1
        e = self.i
        while e > s and _isspace(self.t[e - 1]):
            e -= 1
        return _expand(self.t[s:e])

    def string(self, may_continue=True):
        """A quoted string; returns (text, continued on the next line?). Keys and include names
        may not continue."""
        self.skip()
        if self.peek() != '"':
            raise ConfigError('expected "')
        self.i += 1
        s, esc = self.i, False
        while self.i < len(self.t) and (esc or self.t[self.i] != '"'):
            esc = (not esc and self.t[self.i] == "\\")
            self.i += 1
        if self.i >= len(self.t):
            raise ConfigError("unexpected end of line")
        text = _expand(self.t[s:self.i])
        self.i += 1
        self.skip()
        if self.peek() == "\\":
            if not may_continue:
                raise ConfigError("unexpected \\")
            self.i += 1
            self.skip()
            if self.peek() in ("\0", "!"):
                return text, True
            raise ConfigError("expected end of line after \\")
        return text, False

    def key(self):
        self.skip()
        if self.peek() == '"':  # a quoted key is followed by the data itself, with no ==
            return self.string(False)[0]
        words = []
        w = self.word()
        while w and w != "==":
            words.append(w)
            w = self.word()
        return " ".join(words)


def read_mf(source, filename="<string>", _depth=0, _root=None):
    """Parse `.mf` text (or a path when `source` names an existing file) into a Node tree."""
    if _root is None and os.path.exists(str(source)) and "\n" not in str(source):
        filename = str(source)
        source = open(source).read()
    root = _root if _root is not None else Node()
    stack = [root]
    last = None
    state = "key"
    for line_no, raw in enumerate(source.split("\n"), 1):
        ln = _Line(raw)
        try:
            ln.skip()
            if ln.peek() == "#":
                ln.i += 1
                directive = ln.word()
                if directive != "include":
                    raise ConfigError("unknown directive")
                if _depth > 100:
                    raise ConfigError("include depth too large, probably recursive include")
                name, _ = ln.string(False)
                path = name if os.path.isabs(name) else os.path.join(os.path.dirname(os.path.abspath(filename)), name)
                if not os.path.exists(path):
                    raise ConfigError(f"cannot open include file {name}")
                read_mf(open(path).read(), path, _depth + 1, stack[-1])
                ln.skip()
                if ln.peek() != "\0":
                    raise ConfigError("expected end of line")
                continue
            while True:
                ln.skip()
                if ln.peek() in ("\0", "!"):
                    if state == "data":
                        state = "key"
                    break
                c = ln.peek()
                if state == "key":
                    if c == "{":
                        if last is None:
                            raise ConfigError("unexpected {")
                        stack.append(last)
                        last = None
                        ln.i += 1
                    elif c == "}":
                        if len(stack) <= 1:
                            raise ConfigError("unmatched }")
                        stack.pop()
                        last = None
                        ln.i += 1
                    else:
                        last = stack[-1].add(ln.key())
                        state = "data"
                elif state == "data":
                    if c == "{":
                        stack.append(last)
                        last = None
                        ln.i += 1
                        state = "key"
                    elif c == "}":
                        if len(stack) <= 1:
                            raise ConfigError("unmatched }")
                        stack.pop()
                        last = None
                        ln.i += 1
                        state = "key"
                    elif c == '"':
                        last.value, more = ln.string()
                        state = "cont" if more else "key"
                    else:
                        last.value = ln.rest()
                        state = "key"
                else:  # continuation of a quoted string
                    if c != '"':
                        raise ConfigError('expected " after \\ in previous line')
                    text, more = ln.string()
                    last.value += text
                    state = "cont" if more else "key"
        except ConfigError as e:
            raise ConfigError(f"{filename}:{line_no}: {e}") from None
    if len(stack) != 1:
        raise ConfigError(f"{filename}: unmatched {{")
    return root


# ------------------------------------------------------------------------------- time
_UNITS = {"seconds": 1.0, "second": 1.0, "secs": 1.0, "sec": 1.0, "s": 1.0,
          "minutes": 60.0, "minute": 60.0, "mins": 60.0, "min": 60.0, "m": 60.0,
          "hours": 3600.0, "hour": 3600.0, "hrs": 3600.0, "hr": 3600.0, "h": 3600.0}


def _calendar(fmt, text):
    """std::get_time with `fmt`: a naive calendar time, or None when `text` does not start with
    a time in that format (characters after the time are ignored, as get_time leaves them)."""
    text = text.strip()
    try:
        return datetime.datetime.strptime(text, fmt)
    except ValueError as e:
        msg = str(e)
        if msg.startswith("unconverted data remains: "):
            rest = msg[len("unconverted data remains: "):]
            try:
                return datetime.datetime.strptime(text[:len(text) - len(rest)], fmt)
            except ValueError:
                return None
        return None


class TimeParser:
    """Times in user units (TimeParser.cpp:44-134): a number times the unit factor, hours
    unless `time unit` says otherwise (a named unit or a factor). With a `time format`, a time
    written in that format counts in seconds from `time zero`. The difference is calendar
    arithmetic, which is what mktime gives for times without daylight saving. Anything else
    falls back to a number. A parser for a nested section inherits the format and time zero.
    The reference requires `time zero` again in every such section, or its read throws."""

    def __init__(self, conf, parent=None):
        self.factor = parent.factor if parent else 3600.0
        self.fmt = parent.fmt if parent else ""
        self.zero = parent.zero if parent else None
        if conf is not None:
            fmt = conf.get("time format", self.fmt)
            if fmt:
                zero_text = conf.get("time zero", "")
                if zero_text or self.zero is None or fmt != self.fmt:
                    if not zero_text:
                        raise ConfigError("a `time format` needs a `time zero`")
                    zero = _calendar(fmt, zero_text)
                    if zero is None:
                        raise ConfigError(f"time zero {zero_text!r} does not match the format {fmt!r}")
                    self.zero = zero
                self.fmt = fmt
            u = conf.get("time unit", "default")
            if u in _UNITS:
                self.factor = _UNITS[u]
            elif u != "default":
                try:
                    self.factor = float(u)
                except ValueError:
                    raise ConfigError(f"unknown time unit {u!r}") from None

    def parse(self, s):
        if self.fmt:
            t = _calendar(self.fmt, s)
            if t is not None:
                return (t - self.zero).total_seconds()
        try:
            return float(s) * self.factor
        except ValueError:
            raise ConfigError(f"cannot read {s!r} as a time") from None


def _floats(s, n=None):
    vals = [float(x) for x in re.split(r"[,\s]+", s.strip()) if x]
    if n is not None and len(vals) != n:
        raise ConfigError(f"expected {n} numbers in {s!r}")
    return vals


# ------------------------------------------------------------------------------- WKT
_WKT_TOKEN = re.compile(r"\s*(?:([A-Za-z]+)|([-+]?(?:\d+\.?\d*|\.\d+)(?:[eE][-+]?\d+)?)|([(),]))")
_WKT_KINDS = ("multilinestring", "multipolygon", "multipoint", "linestring", "polygon", "point")


def read_wkt(text):
    """Geometries of a WKT string, as the reference's grammar reads them
    (Geometry/GeometryParser.hpp:92-222): a comma-separated list of POINT, MULTIPOINT,
    LINESTRING, MULTILINESTRING, POLYGON and MULTIPOLYGON, tags in any case with optional Z and
    M, coordinates separated by spaces and points by commas. Returns (kind, has_z, has_m,
    coordinates) tuples: a point is a list of numbers, a line string a list of points, a polygon
    or multi line string a list of line strings, a multi polygon a list of polygons."""
    toks, pos = [], 0
    while pos < len(text):
        if not text[pos:].strip():
            break
        m = _WKT_TOKEN.match(text, pos)
        if not m:
            raise ConfigError(f"failed to parse WKT at {text[pos:]!r}")
        toks.append(("w", m.group(1).lower()) if m.group(1) else (("n", float(m.group(2))) if m.group(2)
                                                                    else ("p", m.group(3))))
        pos = m.end()
    i = 0

    def peek():
        return toks[i] if i < len(toks) else ("end", None)

    def expect(v):
        nonlocal i
        if peek() != ("p", v):
            raise ConfigError(f"failed to parse WKT: expected {v!r}")
        i += 1

    def seq(item):  # '(' item (',' item)* ')'
        nonlocal i
        expect("(")
        out = [item()]
        while peek() == ("p", ","):
            i += 1
            out.append(item())
        expect(")")
        return out

    def coords():  # numbers separated by spaces
        nonlocal i
        out = []
        while peek()[0] == "n":
            out.append(peek()[1])
            i += 1
        if not out:
            raise ConfigError("failed to parse WKT: expected a coordinate")
        return out

    def point_text():
        expect("(")
        c = coords()
        expect(")")
        return c

    def line_text():
        return seq(coords)

    def multiline_text():
        return seq(line_text)

    body = {"point": point_text, "multipoint": lambda: seq(point_text), "linestring": line_text,
            "multilinestring": multiline_text, "polygon": multiline_text,
            "multipolygon": lambda: seq(multiline_text)}

    def geometry():
        nonlocal i
        t = peek()
        if t[0] != "w":
            raise ConfigError("failed to parse WKT: expected a geometry tag")
        word = t[1]
        kind = next((k for k in _WKT_KINDS if word.startswith(k)), None)
        if kind is None:
            raise ConfigError(f"failed to parse WKT: unknown geometry {word!r}")
        i += 1
        flags = word[len(kind):]
        while peek()[0] == "w":  # Z and M may stand apart from the tag
            flags += peek()[1]
            i += 1
        if flags not in ("", "z", "m", "zm"):
            raise ConfigError(f"failed to parse WKT: bad dimension {flags!r}")
        return kind, "z" in flags, "m" in flags, body[kind]()

    geoms = [geometry()]
    while peek() == ("p", ","):
        i += 1
        geoms.append(geometry())
    if i != len(toks):
        raise ConfigError("failed to parse WKT: trailing text")
    return geoms


# -------------------------------------------------------------------------- the model
class Model:
    """A configured solve: mesh, time parameters, scheme, fields, source terms and
    boundaries read from a deck."""

    def __init__(self, tree, base_path="."):
        self.tree = tree
        self.base = base_path
        mesh = tree.child("mesh")
        if mesh is None:
            raise ConfigError("missing `mesh` section")
        self.nx, self.ny = [int(v) for v in _floats(mesh.get("cell count"), 2)]
        self.dx, self.dy = _floats(mesh.get("cell size"), 2)
        self.origin = tuple(_floats(mesh.get("origin", "0.0, 0.0"), 2))
        if float(mesh.get("angle", "0.0")) != 0.0:
            raise ConfigError("rotated meshes are not supported")
        scheme = tree.child("scheme")
        if scheme is None:
            raise ConfigError("missing `scheme` section")
        if (scheme.value or "runge-kutta") != "runge-kutta":
            raise ConfigError(f"unknown scheme type {scheme.value!r}")
        self.parser = TimeParser(scheme)
        self.start_time = self.parser.parse(scheme.get("start time", "0"))
        self.end_time = self.parser.parse(scheme.get("end time"))
        sd = self.parser.parse(scheme.get("step duration", "0"))
        self.step_duration = sd if sd != 0.0 else float(scheme.get("step duration seconds", "60"))
        self.initial_timestep = float(scheme.get("initial timestep seconds", "1.0"))
        self.method = scheme.get("method", "classic")
        self._series = {}
        self._rasters = {}
        self.source_terms = [n for n in tree.equal_range("source term")]
        self.boundaries = [n for n in tree.equal_range("boundary")]
        kinds = [b.value for b in self.boundaries]
        for k in kinds:
            if k not in ("discharge", "head", "stage"):
                raise ConfigError(f"unknown boundary type {k!r}")
        if "head" in kinds and "stage" in kinds:
            raise ConfigError("a head and a stage boundary together are not supported")
        hs = [i for i, k in enumerate(kinds) if k in ("head", "stage")]
        ds = [i for i, k in enumerate(kinds) if k == "discharge"]
        self.head_first = bool(hs and ds and hs[0] < ds[0])
        names = [s.value for s in self.source_terms]
        for n in names:
            if n not in ("manning roughness", "infiltration", "energy loss", "eddy viscosity"):
                raise ConfigError(f"source term {n!r} is not supported")
        self.manning = "manning roughness" in names
        self.eloss_first = ("energy loss" in names and self.manning and
                            names.index("energy loss") < names.index("manning roughness"))
        momentum = {"manning roughness": "manning", "energy loss": "energy loss", "eddy viscosity": "eddy viscosity"}
        self.term_order = [momentum[n] for n in names if n in momentum]
        # EddyViscositySourceTerm::create_source_term (EddyViscositySourceTerm.cpp:112-137)
        self.eddy = None
        for st in self.source_terms:
            if st.value != "eddy viscosity":
                continue
            vt = st.get("viscosity type", "constant")
            if vt == "constant":
                self.eddy = ("constant", float(st.get("default mu", "1.0")))
            elif vt == "smagorinsky":
                self.eddy = ("smagorinsky", float(st.get("constant coefficient", "0.05")),
                             float(st.get("dynamic coefficient", "0.5")))
            else:
                raise ConfigError(f"unknown viscosity type {vt!r}")

    # --- selections and fields
    def selection(self, conf):
        """Cell indices of a MeshSelection (None = global)."""
        kind = conf.value if conf is not None else ""
        if kind in ("", "global"):
            return None
        if kind == "id list":
            ids = [int(n.value) for n in conf.equal_range("id")]
            for n in conf.equal_range("ids"):
                ids += [int(x) for x in _floats(n.value)]
            ids = sorted(set(i for i in ids if 0 <= i < self.nx * self.ny))
            return np.asarray(ids, dtype=np.int64)
        if kind == "at":
            return self._at_selection(conf)
        raise ConfigError(f"unknown mesh selection method {kind!r}")

    def _at_selection(self, conf):
        """MeshSelection "at" (Mesh/MeshSelection.cpp:172-178): the cells containing the points
        of the `wkt` geometry collection (Cartesian2DMesh::get_nearest_object_index); points
        outside the mesh select nothing. Other geometry types cannot select cells, as in the
        reference (MeshSelection.cpp:115-128)."""
        if conf.child("wkt") is None:
            if conf.child("source") is not None:
                raise ConfigError("geometry from a vector file needs GDAL, which is not available")
            return np.zeros(0, dtype=np.int64)
        cells = set()
        for kind, _, _, c in read_wkt(conf.get("wkt")):
            if kind != "point":
                raise ConfigError(f"cannot select cells with a {kind} geometry")
            if len(c) < 2:
                raise ConfigError("a point needs x and y")
            cx = (c[0] - self.origin[0]) * (1.0 / self.dx)
            cy = (c[1] - self.origin[1]) * (1.0 / self.dy)
            if 0.0 <= cx < self.nx and 0.0 <= cy < self.ny:
                cells.add(int(cy) * self.nx + int(cx))
        return np.asarray(sorted(cells), dtype=np.int64)

    def _assign(self, f, sel, v):
        """field *= 0 then += v on the selection (load_constant_input_field,
        FieldGenerator.cpp:43-57): a NaN or infinite value stays NaN."""
        idx = slice(None) if sel is None else sel
        f[idx] = f[idx] * 0.0 + v

    def _load_input(self, f, spec):
        """load_input_field (FieldGenerator.cpp:104-135) into the flat field `f`, in place."""
        sel = self.selection(spec.child("within"))
        kind = (spec.value or "").lower()
        if kind == "composite":  # FieldGenerator.cpp:26-41, ConstantFieldGeneratorModel
            if sel is not None:
                raise ConfigError("composite input fields need a global selection")
            for m in spec.equal_range("model"):
                if m.value != "constant":
                    raise ConfigError(f"unknown field model type {m.value!r}")
                self._assign(f, self.selection(m.child("cells")), float(m.get("value")))
        elif kind == "slope":
            if sel is not None:
                raise ConfigError("sloped input fields need a global selection")
            ox, oy, oz = _floats(spec.get("origin"), 3)
            sx, sy = _floats(spec.get("slope"), 2)
            i = np.arange(self.nx * self.ny)
            x = self.origin[0] + ((i % self.nx) + 0.5) * self.dx + ((i // self.nx) + 0.5) * 0.0
            y = self.origin[1] + ((i % self.nx) + 0.5) * 0.0 + ((i // self.nx) + 0.5) * self.dy
            f[:] = oz + sx * (x - ox) + sy * (y - oy)
        elif kind == "raster":
            r = self.raster(spec.get("name"))
            f[:] = r.map_to_mesh(self.nx, self.ny, self.dx, self.dy, self.origin, cells=sel, field=f).reshape(-1)
        else:
            if kind == "constant":
                v = float(spec.get("value"))
            else:
                try:
                    v = float(kind)
                except ValueError:
                    raise ConfigError(f"{kind!r} is not a known input field specifier") from None
            self._assign(f, sel, v)
        return f

    def raster(self, name):
        """RasterDatabase::get_raster_field_ptr (Raster.cpp:35-68): the `raster field == name`
        section's file, NIMROD only (GDAL is not available)."""
        if name in self._rasters:
            return self._rasters[name]
        conf = next((n for n in self.tree.equal_range("raster field") if n.value == name), None)
        if conf is None:
            raise ConfigError(f"could not find raster field {name!r}")
        src = conf.get("source").lower()
        if src == "gdal":
            raise ConfigError(f"raster field {name!r}: GDAL rasters are not supported (no GDAL)")
        if src != "nimrod":
            raise ConfigError(f"unknown source type {src!r} for raster field {name!r}")
        boxes = conf.equal_range("bbox")
        if len(boxes) > 1:
            raise ConfigError("only one bounding box can be applied to a NIMROD data file")
        fn = conf.get("filename", ".")
        path = fn if os.path.isabs(fn) else os.path.join(self.base, fn)
        try:
            r = NimrodRaster(path, bbox=_floats(boxes[0].value, 4) if boxes else None)
        except (OSError, RasterError) as e:
            raise ConfigError(f"raster field {name!r}: {e}") from None
        self._rasters[name] = r
        return r

    def field(self, name, init):
        """FieldGenerator (FieldGenerator.cpp:137-178): the initial value, then each `set`,
        `add` or `multiply` of the `field == name` section in order; `add` loads its input
        into zeros and `multiply` into ones."""
        f = np.full(self.nx * self.ny, float(init))
        for conf in self.tree.equal_range("field"):
            if conf.value != name:
                continue
            for key, spec in conf:
                if key == "set":
                    self._load_input(f, spec)
                elif key == "add":
                    f = f + self._load_input(np.zeros(self.nx * self.ny), spec)
                elif key == "multiply":
                    f = f * self._load_input(np.ones(self.nx * self.ny), spec)
                else:
                    raise ConfigError(f"unknown field operation {key!r}")
        return f.reshape(self.ny, self.nx)

    # --- time series
    def series(self, name):
        if name in self._series:
            return self._series[name]
        conf = next((n for n in self.tree.equal_range("time series") if n.value == name), None)
        if conf is None:
            raise ConfigError(f"could not find time series {name!r}")
        src = conf.get("source", "not specified").lower()
        if src == "inline":
            sconf = conf.child("source")
            tp = TimeParser(sconf, self.parser)
            data = sconf.child("data")
            if data is None:
                raise ConfigError(f"time series {name!r}: inline source without data")
            times, values = [], []
            for k, n in data:
                t = tp.parse(k.lower())
                if times and t <= times[-1]:
                    raise ConfigError("times in time series must increase")
                times.append(t)
                values.append(float(n.value))
        elif src == "csv":
            times, values = self._csv(conf, TimeParser(conf, self.parser))
        else:
            raise ConfigError(f"unknown time series source {src!r}")
        # TimeSeries::apply_transform (TimeSeries.cpp:81-105) with the `transform` section
        tr = conf.child("transform")
        if tr is not None:
            tf, to = float(tr.get("time factor", "1.0")), float(tr.get("time offset", "0.0"))
            vf, vo = float(tr.get("value factor", "1.0")), float(tr.get("value offset", "0.0"))
            times = [(t + to) * tf for t in times]
            values = [(v + vo) * vf for v in values]
        ts = TimeSeries(times, values)
        self._series[name] = ts
        return ts

    def _csv(self, conf, tp):
        """TimeSeries::load_csv (TimeSeries.cpp:209-259) through rapidcsv 8.51 as the reference
        configures it (trimmed cells, comment and empty lines skipped, the default converter):
        the label row is `skip rows` (+1 with headers, so the first row by default), the row-name
        column `skip cols` (-1: none); named or 1-based numbered time and value columns."""
        fn = conf.get("filename")
        path = fn if os.path.isabs(fn) else os.path.join(self.base, fn)
        sep = conf.get("separator", ",")[:1] or ","
        comment = conf.get("comment character", "#")[:1] or "#"
        headers = conf.get("headers", "true").lower() in ("true", "1", "yes")
        label_row = int(conf.get("skip rows", "-1")) + (1 if headers else 0)
        name_col = int(conf.get("skip cols", "-1"))
        with open(path, "rb") as f:
            rows = rapidcsv_rows(f.read(), sep, comment)
        if headers:
            labels = {}
            if 0 <= label_row < len(rows):
                for i, name in enumerate(rows[label_row]):
                    labels[name] = i  # a repeated label: the last one counts
            cols = []
            for key in ("time column", "value column"):
                name = conf.get(key, "").encode("utf-8").decode("latin-1")
                if name not in labels:
                    raise ConfigError(f"{fn}: no column {conf.get(key, '')!r}")
                cols.append(labels[name])
            tcol, vcol = cols
        else:
            tcol = int(conf.get("time column", "1")) - 1 + name_col + 1
            vcol = int(conf.get("value column", "2")) - 1 + name_col + 1
        body = rows[label_row + 1:] if label_row >= 0 else rows
        times, values = [], []
        for r in body:
            if not (0 <= tcol < len(r) and 0 <= vcol < len(r)):
                raise ConfigError(f"{fn}: a row has no column {max(tcol, vcol) + 1}")
            times.append(tp.parse(r[tcol]))
            values.append(stod_or_nan(r[vcol]))
        return times, values

    # --- building and running
    def build(self, solver_cls, precision="f64", **kw):
        """A solver with the mesh, scheme, fields and source terms of the deck."""
        kwargs = dict(dy=self.dy, rk_method=self.method, step_duration=self.step_duration,
                      initial_dt=self.initial_timestep, manning=self.manning, head_first=self.head_first,
                      eloss_first=self.eloss_first)
        if precision != "f64" or solver_cls.__name__ != "OracleSolver":
            kwargs["precision"] = precision
        kwargs.update(kw)
        s = solver_cls(self.nx, self.ny, self.dx, **kwargs)
        s.set_field("Z", self.field("z_bed", 0.0))
        for f in ("h", "u", "v"):
            s.set_field(f.upper(), self.field(f, 0.0))
        for st in self.source_terms:
            if st.value == "manning roughness":
                # ManningRoughnessSourceTerm.cpp:90-109: defaults, then per-cell fields
                d = (float(st.get("default shallow n", "0.03")), float(st.get("default deep n", "0.3")),
                     float(st.get("default shallow depth", "0.1")), float(st.get("default deep depth", "0.3")))
                s.set_manning(*d)
                for name, fid, dv in (("n_shallow", "N_SHALLOW", d[0]), ("n_deep", "N_DEEP", d[1]),
                                      ("d_shallow", "D_SHALLOW", d[2]), ("d_deep", "D_DEEP", d[3])):
                    if any(c.value == name for c in self.tree.equal_range("field")):
                        s.set_field(fid, self.field(name, dv))
            elif st.value == "infiltration":
                s.set_field("INFIL_RATE", self.field("IR", float(st.get("default infiltration rate", "1e-6"))))
                s.set_field("INFIL_CAP", self.field("IC", float(st.get("default infiltration capacity", "0.1"))))
            elif st.value == "energy loss":
                if st.child("model") is not None:
                    raise ConfigError("energy-loss models are not supported")
                s.set_field("ELOSS_FX", self.field("fdx", float(st.get("default fx/m", "0.0"))))
                s.set_field("ELOSS_FY", self.field("fdy", float(st.get("default fy/m", "0.0"))))
            elif st.value == "eddy viscosity":
                if self.eddy[0] == "constant":
                    s.set_eddy_viscosity("constant", mu=self.eddy[1])
                    if any(c.value == "mu" for c in self.tree.equal_range("field")):
                        s.set_field("EDDY_MU", self.field("mu", self.eddy[1]))
                else:
                    s.set_eddy_viscosity("smagorinsky", mu_const=self.eddy[1], mu_smag=self.eddy[2])
                s.set_source_order(self.term_order)
        return s

    def boundary_values(self, t):
        """start_new_step of every boundary for the step [t, t + L]: per-cell (q0, q1) of the
        discharge boundaries (added) and (h0, h1) of the head or stage boundaries (assigned,
        NaN where unselected), or None when the deck has none."""
        L = self.step_duration
        n = self.nx * self.ny
        q = None
        hb = None
        for b in self.boundaries:
            for key, e in b:
                sel = self.selection(e.child("cells"))
                if key == "constant":
                    v0 = v1 = float(e.get("value"))
                elif key == "time series":
                    ts = self.series(e.get("values"))
                    v0, v1 = ts.at(t), ts.at(t + L)
                else:
                    raise ConfigError(f"unknown boundary entry {key!r}")
                if b.value == "discharge":
                    if q is None:
                        q = (np.zeros(n), np.zeros(n))
                    idx = slice(None) if sel is None else sel
                    q[0][idx] += v0
                    q[1][idx] += v1
                else:
                    if hb is None:
                        hb = (np.full(n, np.nan), np.full(n, np.nan))
                    idx = slice(None) if sel is None else sel
                    hb[0][idx] = v0
                    hb[1][idx] = v1
        return q, hb

    def forcing(self, solver, t):
        """Upload the step's boundary values to `solver` and set its forcing: one uniform
        rain pair when every cell gets the same discharge, per-cell fields otherwise."""
        q, hb = self.boundary_values(t)
        f = Forcing()
        f.rain_kind = RAIN_NONE
        f.head_kind = HEAD_NONE
        if q is not None:
            if np.all(q[0] == q[0][0]) and np.all(q[1] == q[1][0]):
                f.rain_kind, f.rain_q0, f.rain_q1 = RAIN_UNIFORM, float(q[0][0]), float(q[1][0])
            else:
                f.rain_kind = RAIN_FIELDS
        if hb is not None:  # head targets first: a forcing that names them needs them set
            solver.set_field("HBDY0", hb[0].reshape(self.ny, self.nx))
            solver.set_field("HBDY1", hb[1].reshape(self.ny, self.nx))
            f.head_kind = STAGE_FIELDS if any(b.value == "stage" for b in self.boundaries) else HEAD_FIELDS
        solver.set_forcing(f)
        if f.rain_kind == RAIN_FIELDS:  # per-cell discharge after the forcing that clears them
            solver.set_field("QBDY0", q[0].reshape(self.ny, self.nx))
            solver.set_field("QBDY1", q[1].reshape(self.ny, self.nx))
        return f

    # --- outputs and measures
    def _path(self, fn):
        return fn if os.path.isabs(fn) else os.path.join(self.base, fn)

    def outputs(self):
        """make_field_output_file (OutputFile.hpp:229-258) for each enabled `output == name`
        section: the fields named by its `field` keys (the section's name when there are
        none), written from `start time` every `every` (or `every seconds`) to
        `<filename>_<t>.csv`, `filename` defaulting to output/<name> beside the deck. Field
        names the solver does not have are skipped, as in the reference. Only cell outputs
        are written."""
        outs = []
        for conf in self.tree.equal_range("output"):
            name = conf.value
            if conf.get("enabled", "true").strip().lower() in ("false", "0"):
                continue
            at = conf.get("at", "cells")
            if at != "cells":
                raise ConfigError(f"output {name!r}: only cell outputs are supported (at == {at})")
            fields = [f.value for f in conf.equal_range("field")] or [name]
            for f in fields:
                if f in ("mannings_n", "friction_slope"):  # ManningRoughnessSourceTerm.hpp:151-158
                    raise ConfigError(f"output {name!r}: {f!r} is formed inside the stage kernels and not kept")
            fields = [f for f in fields if f in _OUTPUT_FIELDS or f == "stage"]
            start = self.parser.parse(conf.get("start time")) if conf.child("start time") is not None else self.start_time
            if conf.child("every") is not None:
                every = self.parser.parse(conf.get("every"))
            elif conf.child("every seconds") is not None:
                every = float(conf.get("every seconds"))
            else:
                raise ConfigError(f"output {name!r}: needs `every` or `every seconds`")
            out = MultiFieldOutput(self._path(conf.get("filename", os.path.join("output", name))), fields, every,
                                   start, origin=self.origin, delimiter=conf.get("delimiter", ", "))
            outs.append(out)
        return outs

    def measures(self):
        """SaintVenantHPointMeasure::create_measures (SaintVenant/Measure.hpp:214-224): one depth
        measure per `h-point == name` of the `measures` section, at the cell nearest its
        `location`, written to `filename` (default output/measures/<name>.csv beside the deck).
        The reference builds no other measure from a deck."""
        res = []
        mconf = self.tree.child("measures")
        if mconf is None:
            return res
        for conf in mconf.equal_range("h-point"):
            try:
                m = DepthPointMeasure(_floats(conf.get("location"), 2), self.nx, self.ny, self.dx, self.dy,
                                      self.origin, name=conf.value)
            except ValueError as e:
                raise ConfigError(f"measure {conf.value!r}: {e}") from None
            m.filename = self._path(conf.get("filename", os.path.join("output", "measures", conf.value + ".csv")))
            res.append(m)
        return res

    def solve(self, solver, on_step=None, write_outputs=True):
        """TypedTemporalScheme::solve (TemporalScheme.hpp:244-276) over the deck's start and end
        times. Each step begins with the measures (end_of_step, SaintVenant/Solver.hpp:90-98),
        then the outputs (do_outputs, RungeKutta.hpp:444-449), then `on_step`; the outputs run
        once more at the end time. The reference never writes its measures
        (Output/Measure.hpp:87-98 has no caller); here each is written to its file at the end.
        With `write_outputs` false, no file is written."""
        outs = self.outputs() if write_outputs else []
        meas = self.measures() if write_outputs else []
        for m in meas:  # the measures' values (and times) are written in the solver's value type
            m.value_type = np.float64 if getattr(solver, "precision", "f64") == "f64" else np.float32
        n = num_steps(self.start_time, self.end_time, self.step_duration)
        per_step = []
        for i in range(n):
            t = self.start_time + i * self.step_duration
            for m in meas:
                m.update(t, solver)
            for o in outs:
                o.timed_output(t, solver)
            if on_step:
                on_step(t, solver)
            self.forcing(solver, t)
            per_step.append(solver.advance())
        t_end = self.start_time + n * self.step_duration
        for o in outs:
            o.timed_output(t_end, solver)
        if on_step:
            on_step(t_end, solver)
        for m in meas:
            m.write(m.filename)
        return per_step


def load(path):
    """Read a deck; relative file names inside it resolve against its directory."""
    return Model(read_mf(path), base_path=os.path.dirname(os.path.abspath(path)))


__all__ = ["ConfigError", "Node", "read_mf", "read_wkt", "TimeParser", "Model", "load"]
