"""Time series of the configuration decks (mfcm_b200/config.py, mfcm_b200.TimeSeries) against
the reference's own reader (CPU; needs the reference source tree).

oracle/ref_pin/build.py compiles the reference's TimeSeries (src/Input/TimeSeries.cpp) with the
rapidcsv 8.51 it vendors; oracle/ref_pin/refpin.py loads a series through
TimeSeries<double, double>::load and evaluates TimeSeries::at. The same CSV files and inline
data go through both, and the times and values must agree bit for bit (NaN where the
reference's converter gives its default): rapidcsv's cell splitting, quoting, trimming, comment
and empty lines, label row and row-name column, std::stod's prefix parsing and range errors,
and the series' transform. Times are plain numbers of seconds: the reference's time parser is
built on Boost, which is not available. Without the reference tree the tests skip.
"""
import numpy as np
import pytest

from mfcm_b200 import TimeSeries, config
from oracle.ref_pin import refpin

pytestmark = pytest.mark.skipif(not refpin.available(), reason="reference source tree not present")

DECK_HEAD = "mesh\n{\n  cell count == 4 4\n  cell size == 1 1\n}\nscheme == runge-kutta\n{\n  end time == 60\n}\n"
VALUES = ["1.5", " 2e-5 ", "abc", "12abc", "1e-310", "inf", "-inf", "0x10", "0x1.8p1", "1e999", "-0", ".5", "-.5e3",
          '"3.5"', '""', "nan", "1e", "+7", "2.2250738585072011e-308", "4e-320", "0", "", "1,5"]


def _ours(tmp_path, section, data=None, transform=None):
    # times in seconds: the stand-in time parser of the pin reads plain seconds, where the
    # reference's own parser defaults to hours
    lines = ["time series == s", "{", "  time unit == seconds"]
    lines += [f"  {k} == {v}" for k, v in section.items() if k != "source" or not data]
    if data:
        lines += ["  source == inline", "  {", "    time unit == seconds", "    data", "    {"]
        lines += [f"      {t} == {v}" for t, v in data]
        lines += ["    }", "  }"]
    if transform:
        lines += ["  transform", "  {"] + [f"    {k} == {v}" for k, v in transform.items()] + ["  }"]
    lines.append("}")
    deck = tmp_path / "deck.mf"
    deck.write_text(DECK_HEAD + "\n".join(lines) + "\n")
    ts = config.load(str(deck)).series("s")
    return np.array(ts.t), np.array(ts.v)


def _same(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return a.shape == b.shape and np.array_equal(np.isnan(a), np.isnan(b)) and np.array_equal(a[~np.isnan(a)],
                                                                                              b[~np.isnan(b)])


def _csv_case(rng, path, sep, comment, headers, skip_rows, skip_cols):
    """A CSV file with extra columns, comment and empty lines, CRLF endings, quoted and padded
    cells and awkward numbers; returns the section keys."""
    lo = skip_cols + 1 if skip_cols >= 0 else 0     # the columns after the row-name column
    ncols = lo + int(rng.integers(2, 5))
    tcol, vcol = (int(c) for c in rng.choice(np.arange(lo, ncols), 2, replace=False))
    names = [f"c{i}" for i in range(ncols)]
    names[tcol], names[vcol] = "time", "rain"
    out = []
    if rng.uniform() < 0.3:
        out.append(b"\xef\xbb\xbf")
    for _ in range(skip_rows + 1 if skip_rows >= 0 else 0):  # `skip rows` N passes over N + 1 rows
        out.append(("skipped" + sep + "row\n").encode())
    if rng.uniform() < 0.5:
        out.append(f"{comment} a comment\n".encode())
    if headers:
        out.append((sep.join(f" {n} " if rng.uniform() < 0.3 else n for n in names) + "\n").encode())
    t = 0.0
    nrows = int(rng.integers(2, 14))
    for r in range(nrows):
        t += float(rng.choice([0.5, 30.0, 60.0, 900.0]))
        cells = [str(rng.integers(0, 9)) for _ in range(ncols)]
        cells[tcol] = (f" {t:g} " if rng.uniform() < 0.3 else f"{t:g}")
        v = str(rng.choice(VALUES))
        if sep in v and not (v.startswith('"') and v.endswith('"')):
            v = f'"{v}"'
        cells[vcol] = v
        end = "\r\n" if rng.uniform() < 0.3 else "\n"
        if r == nrows - 1 and rng.uniform() < 0.3:
            end = ""
        out.append((sep.join(cells) + end).encode())
        if rng.uniform() < 0.15 and end:
            out.append(b"\n")
        if rng.uniform() < 0.1 and end:
            out.append(f"  {comment} indented comment\n".encode())
    path.write_bytes(b"".join(out))
    section = {"source": "csv", "filename": str(path), "separator": sep, "comment character": comment,
               "headers": "true" if headers else "false"}
    if skip_rows >= 0:
        section["skip rows"] = str(skip_rows)
    if skip_cols >= 0:
        section["skip cols"] = str(skip_cols)
    if headers:
        section["time column"], section["value column"] = "time", "rain"
    else:
        base = skip_cols + 1 if skip_cols >= 0 else 0
        section["time column"], section["value column"] = str(tcol - base + 1), str(vcol - base + 1)
    return section


@pytest.mark.parametrize("seed", range(40))
def test_csv_series_match_reference(tmp_path, seed):
    rng = np.random.default_rng(seed)
    sep = [",", ";", "|", ":"][seed % 4]   # a deck value is trimmed: it cannot hold a blank
    comment = ["#", "%"][seed % 2]
    headers = seed % 3 != 0
    skip_rows = [-1, -1, 0, 1, 2][seed % 5]
    skip_cols = [-1, -1, 0, 1][seed % 4]
    section = _csv_case(rng, tmp_path / "s.csv", sep, comment, headers, skip_rows, skip_cols)
    transform = {"time factor": "60", "value offset": "0.25"} if seed % 7 == 0 else None
    try:
        rt, rv = refpin.ts_load(section, transform=transform)
    except refpin.RefReaderError:
        with pytest.raises(config.ConfigError):
            _ours(tmp_path, section, transform=transform)
        return
    ot, ov = _ours(tmp_path, section, transform=transform)
    assert _same(ot, rt), (ot, rt)
    assert _same(ov, rv), (ov, rv, (tmp_path / "s.csv").read_bytes())


def test_csv_series_reference_rules(tmp_path):
    """The rules the first version of the reader had wrong, each seen in the reference: a line
    of blanks is a row (here one too short to read), `skip cols` offsets numbered columns, a
    repeated label means its last column, and values take std::stod's prefix and range rules."""
    p = tmp_path / "s.csv"
    p.write_bytes(b"time,v,v\n0,1,2\n   \n60,3,4\n")
    sec = {"source": "csv", "filename": str(p), "time column": "time", "value column": "v"}
    with pytest.raises(refpin.RefReaderError):
        refpin.ts_load(sec)
    with pytest.raises(config.ConfigError):
        _ours(tmp_path, sec)
    p.write_bytes(b"time,v,v\n0,1,2\n60,3,4\n")
    rt, rv = refpin.ts_load(sec)
    assert list(rv) == [2.0, 4.0] and _same(_ours(tmp_path, sec)[1], rv)
    p.write_bytes(b"x,0,9,1\ny,60,8,12abc\nz,120,7,1e-310\n")
    sec = {"source": "csv", "filename": str(p), "headers": "false", "skip cols": "0", "time column": "1",
           "value column": "3"}
    rt, rv = refpin.ts_load(sec)
    assert list(rt) == [0.0, 60.0, 120.0] and rv[1] == 12.0 and np.isnan(rv[2])
    ot, ov = _ours(tmp_path, sec)
    assert _same(ot, rt) and _same(ov, rv)


@pytest.mark.parametrize("seed", range(10))
def test_inline_series_and_transform_match_reference(tmp_path, seed):
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(2, 9))
    times = np.cumsum(rng.uniform(0.5, 600.0, n))
    data = [(f"{t:.6g}", f"{v:.9g}") for t, v in zip(times, rng.normal(0.0, 1e-4, n))]
    transform = {}
    if seed % 2:
        transform["time factor"] = str(rng.choice(["60", "3600", "0.5"]))
        transform["value factor"] = str(rng.choice(["2.777777777777778e-07", "0.001", "-1"]))
    if seed % 3 == 0:
        transform["time offset"] = "-30"
        transform["value offset"] = "1e-5"
    rt, rv = refpin.ts_load({"source": "inline"}, data=data, transform=transform or None)
    ot, ov = _ours(tmp_path, {"source": "inline"}, data=data, transform=transform or None)
    assert _same(ot, rt) and _same(ov, rv)


def test_missing_column_name_is_an_error(tmp_path):
    """A finding, fixed here: the reference looks a missing label up as index -1, and with a
    row-name column (`skip cols` 0 or more) that index wraps around to the row-name column, so
    the series silently takes its values from there. The package refuses the deck instead."""
    p = tmp_path / "s.csv"
    p.write_bytes(b"id,time,rain\n10,0,1\n20,60,2\n")
    sec = {"source": "csv", "filename": str(p), "skip cols": "0", "time column": "time", "value column": "flow"}
    rt, rv = refpin.ts_load(sec)
    assert list(rt) == [0.0, 60.0] and list(rv) == [10.0, 20.0]   # the row-name column
    with pytest.raises(config.ConfigError, match="flow"):
        _ours(tmp_path, sec)


def test_interpolation_matches_reference():
    """TimeSeries::at (ts_linterp) below the last knot, before the first one included."""
    rng = np.random.default_rng(7)
    for _ in range(50):
        n = int(rng.integers(2, 12))
        t = np.cumsum(rng.uniform(0.1, 1000.0, n)) - float(rng.uniform(0, 500))
        v = rng.normal(0.0, 1.0, n) * 10.0 ** rng.integers(-8, 3)
        q = np.concatenate([t[:-1], rng.uniform(t[0] - 100.0, t[-1], 40), np.nextafter(t[1:], -np.inf)])
        q = q[q < t[-1]]
        ref = refpin.ts_at(t, v, q)
        ts = TimeSeries(t, v)
        ours = np.array([ts.at(float(x)) for x in q])
        assert np.array_equal(ours.view(np.int64), ref.view(np.int64))
