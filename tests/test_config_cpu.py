"""The `.mf` configuration front end (mfcm_b200/config.py): the reader's grammar and errors,
the time units, the field generators, selections and time series, and a whole deck whose
solve equals the same problem set up through the API, bit for bit (oracle, CPU)."""
import os

import numpy as np
import pytest

from mfcm_b200 import config, solve, TimeSeries, HEAD_FIELDS
from mfcm_b200.config import ConfigError, read_mf
from oracle.sv_oracle_py import OracleSolver
from tests.scenarios import same

DECKS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "decks")


def test_reader_keys_values_nesting_and_repeats():
    t = read_mf('mesh\n{\n  cell count == 10 20   ! trailing comment\n  "quoted key" "a \\"b\\"\\tc"\n}\n'
                'boundary == head\n{\n}\nboundary == stage\n'
                'long == "first part" \\\n        " second"\n')
    mesh = t.child("mesh")
    assert mesh.get("cell count") == "10 20"
    assert mesh.get("quoted key") == 'a "b"\tc'
    assert [n.value for n in t.equal_range("boundary")] == ["head", "stage"]
    assert t.get("long") == "first part second"


def test_reader_errors():
    for bad in ("}\n", "{\n", "a\n{\n", "#define x\n", 'a == "open\n', 'k == "x" \\ y\n',
                '"k" \\\n', 'k == "x" \\\nnext\n'):
        with pytest.raises(ConfigError):
            read_mf(bad)


def test_include_is_relative_to_the_including_file(tmp_path):
    (tmp_path / "sub").mkdir()
    (tmp_path / "sub" / "inner.mf").write_text("x == 1\n")
    (tmp_path / "main.mf").write_text('a\n{\n#include "sub/inner.mf"\n}\n')
    t = read_mf(str(tmp_path / "main.mf"))
    assert t.child("a").get("x") == "1"


def test_time_units():
    assert config.TimeParser(read_mf("")).parse("2") == 7200.0          # hours by default
    assert config.TimeParser(read_mf("time unit == minutes\n")).parse("1.5") == 90.0
    assert config.TimeParser(read_mf("time unit == 10\n")).parse("3") == 30.0
    with pytest.raises(ConfigError):
        config.TimeParser(read_mf("time unit == fortnights\n"))
    with pytest.raises(ConfigError):
        config.TimeParser(read_mf("time format == %Y\n"))


def test_deck_fields_series_and_boundaries():
    m = config.load(os.path.join(DECKS, "catchment.mf"))
    assert (m.nx, m.ny, m.dx, m.step_duration, m.end_time) == (24, 16, 5.0, 30.0, 120.0)
    assert m.series("storm").t == [0.0, 60.0, 90.0, 180.0, 6000.0]      # CSV times in minutes
    z = m.field("z_bed", 0.0)
    assert z[0, 0] == 10.0 + (-0.01) * 2.5 + 0.002 * 2.5
    assert z.ravel()[150] == (10.0 + (-0.01) * 32.5 + 0.002 * 32.5) + 0.75   # the id-list bump
    assert z.ravel()[151] == 10.0 + (-0.01) * 37.5 + 0.002 * 32.5
    q, hb = m.boundary_values(30.0)
    assert q[0][0] == m.series("storm").at(30.0) and q[1][0] == m.series("storm").at(60.0)
    assert np.count_nonzero(~np.isnan(hb[0])) == 16 and np.all(hb[0][23::24] == 0.0)


def test_unsupported_features_are_named():
    base = "mesh\n{\ncell count == 4 4\ncell size == 1 1\n}\nscheme == runge-kutta\n{\nend time == 1\n}\n"
    for extra, what in (("source term == eddy viscosity\n{\nviscosity type == laminar\n}\n", "laminar"),
                        ("boundary == weir\n", "weir")):
        with pytest.raises(ConfigError, match=what):
            config.Model(read_mf(base + extra))
    m = config.Model(read_mf(base + "field == h\n{\nset == raster\n{\nname == dem\n}\n}\n"))
    with pytest.raises(ConfigError, match="raster"):
        m.field("h", 0.0)


def _direct(m, eddy=False):
    """The same problem as catchment.mf, set up through the API (with `eddy`, the constant
    eddy viscosity 0.4 m^2/s, 0.6 on cells 30-32, listed before the roughness term)."""
    o = OracleSolver(m.nx, m.ny, m.dx, m.dy, step_duration=m.step_duration, initial_dt=1.0)
    if eddy:
        mu = np.full(m.nx * m.ny, 0.4)
        mu[30:33] += 0.2
        o.set_field("EDDY_MU", mu.reshape(m.ny, m.nx))
        o.set_eddy_viscosity("constant", mu=0.4)
        o.set_source_order(["eddy viscosity", "manning"])
    o.set_field("Z", m.field("z_bed", 0.0))
    o.set_field("H", np.full((m.ny, m.nx), 0.002))
    o.set_field("U", np.zeros((m.ny, m.nx)))
    o.set_field("V", np.zeros((m.ny, m.nx)))
    o.set_manning(0.035, 0.035, 0.1, 0.3)
    storm = TimeSeries([0.0, 60.0, 90.0, 180.0, 6000.0], [1e-5, 2e-5, 2e-5, 0.0, 0.0])
    hb = np.full((m.ny, m.nx), np.nan)
    hb[:, -1] = 0.0
    o.set_field("HBDY0", hb)
    o.set_field("HBDY1", hb)
    for i in range(4):
        t = 30.0 * i
        from mfcm_b200 import Forcing, RAIN_UNIFORM
        f = Forcing()
        f.rain_kind, f.rain_q0, f.rain_q1 = RAIN_UNIFORM, storm.at(t), storm.at(t + 30.0)
        f.head_kind = HEAD_FIELDS
        o.set_forcing(f)
        o.advance()
    return o


def test_deck_solve_equals_the_api_setup():
    m = config.load(os.path.join(DECKS, "catchment.mf"))
    a = m.build(OracleSolver)
    m.solve(a)
    b = _direct(m)
    for f in ("H", "U", "V"):
        assert same(a.get_field(f), b.get_field(f)), f
    assert a.stats() == b.stats()
    assert a.stats()["accepted"] > 0 and a.stats()["outflow"] > 0.0


def test_inline_series_multiply_and_infiltration_deck():
    deck = read_mf("""
mesh
{
  cell count == 6 4
  cell size == 2 2
}
scheme == runge-kutta
{
  time unit == minutes
  end time == 2
  step duration == 1
}
time series == pulse
{
  source == inline
  {
    time unit == seconds
    data
    {
      0 == 0.0
      30 == 3e-5
      90 == 0
    }
  }
}
field == z_bed
{
  set == 1.0
  multiply == 2.5
  {
    within == id list
    {
      ids == 0 1 2
    }
  }
  add == constant
  {
    value == 0.25
  }
}
field == IR
{
  set == 1e-6
}
field == IC
{
  set == 5e-4
}
source term == infiltration
boundary == discharge
{
  time series == rain
  {
    values == pulse
  }
}
""")
    m = config.Model(deck)
    assert (m.end_time, m.step_duration) == (120.0, 60.0)
    ts = m.series("pulse")
    assert ts.t == [0.0, 30.0, 90.0] and abs(ts.at(60.0) - 1.5e-5) < 1e-20
    z = m.field("z_bed", 0.0).ravel()
    assert list(z[:4]) == [2.75, 2.75, 2.75, 1.25]
    a = m.build(OracleSolver)
    m.solve(a)
    ic = a.get_field("INFIL_CAP")
    assert np.all(ic < 5e-4) and np.all(ic >= 0.0)       # capacity consumed as it infiltrates


def test_eddy_viscosity_deck_equals_the_api_setup():
    text = open(os.path.join(DECKS, "catchment.mf")).read().replace(
        "source term == manning roughness",
        "source term == eddy viscosity\n{\n  viscosity type == constant\n  default mu == 0.4\n}\n"
        "field == mu\n{\n  set == 0.4\n  add == 0.2\n  {\n    within == id list\n    {\n      ids == 30 31 32\n"
        "    }\n  }\n}\nsource term == manning roughness")
    m = config.Model(read_mf(text, filename=os.path.join(DECKS, "catchment.mf")), base_path=DECKS)
    assert m.eddy == ("constant", 0.4) and m.term_order == ["eddy viscosity", "manning"]
    a = m.build(OracleSolver)
    m.solve(a)
    b = _direct(m, eddy=True)
    for f in ("H", "U", "V"):
        assert same(a.get_field(f), b.get_field(f)), f
    plain = _direct(m)
    assert not same(a.get_field("U"), plain.get_field("U"))


def test_deck_outputs_and_measures(tmp_path):
    """Output sections write timed CSV files of the named cell fields; an h-point measure records
    the depth of the cell nearest its location at the start of every step."""
    text = open(os.path.join(DECKS, "catchment.mf")).read() + """
output == state
{
  field == h
  field == stage
  field == no such field
  every seconds == 60
  delimiter == ;
  filename == out/state
}
output == quiet
{
  enabled == false
  every seconds == 30
}
measures
{
  h-point == gauge
  {
    location == 62.5 42.5
  }
}
"""
    (tmp_path / "deck.mf").write_text(text)
    for extra in ("boundaries.mf", "storm.csv"):
        (tmp_path / extra).write_text(open(os.path.join(DECKS, extra)).read())
    m = config.load(str(tmp_path / "deck.mf"))
    seen = []
    s = m.build(OracleSolver)
    m.solve(s, on_step=lambda t, x: seen.append((t, x.get_field("H").ravel()[8 * 24 + 12])))
    files = sorted(p.name for p in (tmp_path / "out").iterdir())
    assert files == ["state_0.000000.csv", "state_120.000000.csv", "state_60.000000.csv"]
    lines = (tmp_path / "out" / "state_120.000000.csv").read_text().splitlines()
    assert lines[0] == 'X;Y;"h";"stage";'
    h = s.get_field("H").ravel()
    z = s.get_field("Z").ravel()
    assert lines[1] == f"2.5;2.5;{h[0]:f};{z[0] + h[0]:f};"
    assert not (tmp_path / "output" / "quiet_0.000000.csv").exists()
    gauge = (tmp_path / "output" / "measures" / "gauge.csv").read_text().splitlines()
    assert gauge[0] == '"ID", "gauge", ' and len(gauge) == 1 + 4      # steps at 0, 30, 60, 90 s
    assert [float(r.split(",")[1]) for r in gauge[1:]] == [round(v, 6) for t, v in seen[:4]]


def test_wkt_reader():
    g = config.read_wkt("POINT (1 2), point z(1 2 3), MULTIPOINT ((1 2), (3 4)), LINESTRING (0 0, 1 1),"
                        " POLYGON ((0 0, 4 0, 4 4, 0 0)), MULTIPOLYGON (((0 0, 1 0, 0 1, 0 0))), Point ZM (1 2 3 4)")
    assert [x[0] for x in g] == ["point", "point", "multipoint", "linestring", "polygon", "multipolygon", "point"]
    assert g[1][1:] == (True, False, [1.0, 2.0, 3.0]) and g[6][1:3] == (True, True)
    assert g[4][3] == [[[0.0, 0.0], [4.0, 0.0], [4.0, 4.0], [0.0, 0.0]]]
    for bad in ("POINT (1 2", "CIRCLE (1 2)", "POINT Q (1 2)", "POINT (1 2) junk", "POINT ()", "MULTIPOINT (1 2)"):
        with pytest.raises(ConfigError):
            config.read_wkt(bad)


def test_point_selections():
    base = ("mesh\n{\ncell count == 24 16\ncell size == 5 5\n}\nscheme == runge-kutta\n{\nend time == 1\n}\n"
            "field == z_bed\n{\n  set == 1.0\n  add == constant\n  {\n    value == 0.5\n    within == at\n    {\n"
            "      wkt == %s\n    }\n  }\n}\n")
    m = config.Model(read_mf(base % "POINT (12.5 7.5), POINT (1000 1000), POINT Z (2.5 2.5 9)"))
    z = m.field("z_bed", 0.0).ravel()
    assert list(np.flatnonzero(z != 1.0)) == [0, 26] and z[26] == 1.5      # (1000, 1000) is outside
    m = config.Model(read_mf(base % "LINESTRING (0 0, 10 10)"))
    with pytest.raises(ConfigError, match="linestring"):
        m.field("z_bed", 0.0)


def test_calendar_times(tmp_path):
    """A `time format` makes times calendar times counted from `time zero`; nested sections
    (a CSV time series here) inherit the format and the time zero; plain numbers still count
    in the unit."""
    (tmp_path / "rain.csv").write_text("when,rate\n2023-03-01 00:00,1e-5\n2023-03-01 00:30,3e-5\n"
                                       "2023-03-01 02:00,0\n")
    deck = tmp_path / "deck.mf"
    deck.write_text("""
mesh
{
  cell count == 4 4
  cell size == 1 1
}
scheme == runge-kutta
{
  time format == %Y-%m-%d %H:%M
  time zero == 2023-03-01 00:00
  start time == 2023-03-01 00:10
  end time == 2023-03-01 01:10
  step duration == 0.5
}
time series == rain
{
  source == csv
  filename == rain.csv
  time column == when
  value column == rate
}
""")
    m = config.load(str(deck))
    assert (m.start_time, m.end_time, m.step_duration) == (600.0, 4200.0, 1800.0)
    ts = m.series("rain")
    assert ts.t == [0.0, 1800.0, 7200.0] and ts.v == [1e-5, 3e-5, 0.0]
    with pytest.raises(ConfigError, match="time zero"):
        config.TimeParser(read_mf("time format == %Y-%m-%d\n"))


def test_output_field_names():
    base = ("mesh\n{\ncell count == 4 4\ncell size == 1 1\n}\nscheme == runge-kutta\n{\nend time == 1\n}\n"
            "output == o\n{\nfield == %s\nevery seconds == 10\n}\n")
    assert [o.fields for o in config.Model(read_mf(base % "fx")).outputs()] == [["fx"]]
    assert [o.fields for o in config.Model(read_mf(base % "nothing")).outputs()] == [[]]   # skipped, as there
    with pytest.raises(ConfigError, match="friction_slope"):
        config.Model(read_mf(base % "friction_slope")).outputs()
