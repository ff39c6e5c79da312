"""Outputs, measures and checkpoints (mfcm_b200/outputs.py) on the CPU: the CSV text matches
what the reference's C++ writes (std::to_string for values, ostream << for coordinates,
checked against a compiled C++ program), the raw binary layout, the output schedule, the
point measure, and a checkpoint that resumes the oracle bit for bit."""
import os
import struct
import subprocess

import numpy as np
import pytest

from mfcm_b200 import outputs, synth, solve, EDGE_XMAX
from oracle.sv_oracle_py import OracleSolver
from tests.scenarios import same, rain_series

VALUES = [0.0, -0.0, 0.5, 1e-7, -3.25, 123456.789, 1e-300, 2.5e6, 1.0 / 3.0, -7.0e-5, 9.999995e-7, 1e21]


def test_formatting_matches_the_cpp_library(tmp_path):
    src = tmp_path / "fmt.cpp"
    src.write_text("#include <cstdio>\n#include <iostream>\n#include <string>\n#include <cstdlib>\n"
                   "int main(int argc, char** argv) {\n"
                   "  for (int i = 1; i < argc; ++i) {\n"
                   "    double x = std::strtod(argv[i], nullptr);\n"
                   "    std::cout << std::to_string(x) << ' ' << x << '\\n';\n"
                   "  }\n}\n")
    exe = tmp_path / "fmt"
    subprocess.run(["g++", "-O0", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)] + [repr(v) for v in VALUES], capture_output=True, text=True,
                         check=True).stdout.split("\n")
    for v, line in zip(VALUES, out):
        a, b = line.split(" ")
        assert outputs.fmt_value(v) == a, v
        assert outputs.fmt_coord(v) == b, v


def test_csv_layout():
    text = outputs.csv_text(["h", "u"], [[0.5, -0.0], [1e-7, 123456.789]], locations=([1.0, 2.5e6], [0.5, 1.5]))
    assert text == ('X, Y, "h", "u", \n'
                    '1, 0.5, 0.500000, 0.000000, \n'
                    '2.5e+06, 1.5, -0.000000, 123456.789000, \n')


def test_raw_binary_layout_and_round_trip():
    cols = [np.arange(5.0), np.linspace(-1, 1, 5)]
    data = outputs.raw_binary_bytes(cols, np.float32)
    assert struct.unpack_from("<QQQ", data) == (5, 2, 4)
    assert len(data) == 24 + 5 * 2 * 4
    arr, n = outputs.read_raw_binary(data)
    assert n == len(data)
    assert np.array_equal(arr[:, 1], np.float32(cols[1]))   # row-major: row r = (col0[r], col1[r])
    assert np.array_equal(np.frombuffer(data[24:32], np.float32), [0.0, -1.0])


class _Stub:
    nx, ny, dx, dy = 3, 2, 2.0, 5.0

    def get_field(self, name):
        return {"H": np.arange(6.0).reshape(2, 3), "Z": np.full((2, 3), 10.0)}[name]


def test_timed_multi_field_output(tmp_path):
    o = outputs.MultiFieldOutput(str(tmp_path / "out" / "depth"), ["h", "stage"], every=600.0)
    for t in (0.0, 300.0, 600.0, 900.0, 1250.0):
        o.timed_output(t, _Stub())
    assert [os.path.basename(p) for p in o.written] == ["depth_0.000000.csv", "depth_600.000000.csv",
                                                       "depth_1250.000000.csv"]
    lines = open(o.written[0]).read().splitlines()
    assert lines[0] == 'X, Y, "h", "stage", '
    assert lines[1] == "1, 2.5, 0.000000, 10.000000, "       # cell 0 centre (0.5 dx, 0.5 dy)
    assert lines[6] == "5, 7.5, 5.000000, 15.000000, "


def test_depth_point_measure_picks_the_containing_cell(tmp_path):
    m = outputs.DepthPointMeasure((4.1, 6.0), 3, 2, 2.0, 5.0)
    assert m.index == 1 * 3 + 2
    m.update(0.0, _Stub())
    m.write(str(tmp_path / "pt.csv"))
    assert open(tmp_path / "pt.csv").read() == '"ID", "h_point", \n0.000000, 5.000000, \n'
    with pytest.raises(ValueError):
        outputs.DepthPointMeasure((6.5, 1.0), 3, 2, 2.0, 5.0)


def _oracle(nx, ny, dx, z):
    o = OracleSolver(nx, ny, dx, cn_target=0.5, step_duration=20.0, rain_mode="physical")
    o.set_field("Z", z)
    o.set_manning(0.03, 0.03, 0.1, 0.3)
    return o


def test_checkpoint_resumes_the_oracle_bit_for_bit(tmp_path):
    nx, ny, dx = 30, 20, 4.0
    z = synth.plane_with_gaussians(nx, ny, dx, seed=2)
    rain = rain_series(60 * synth.MM_PER_H, stop=1e4)
    a = _oracle(nx, ny, dx, z)
    a.set_field("H", np.full((ny, nx), 2e-3))
    solve(a, 0.0, 40.0, rain=rain, head=0.0, head_edges=EDGE_XMAX)
    ck = str(tmp_path / "ck.bin")
    outputs.save_checkpoint(a, ck, t=40.0)
    solve(a, 40.0, 80.0, rain=rain, head=0.0, head_edges=EDGE_XMAX)
    b = _oracle(nx, ny, dx, z)
    meta = outputs.load_checkpoint(b, ck)
    assert meta["t"] == 40.0
    solve(b, 40.0, 80.0, rain=rain, head=0.0, head_edges=EDGE_XMAX)
    for f in ("H", "U", "V"):
        assert same(a.get_field(f), b.get_field(f)), f
    sa, sb = a.stats(), b.stats()
    assert sa == sb
