"""The C++ facade (include/mfcm_b200.hpp): classes named after the reference's
(Cartesian2DMesh, SaintVenantSolver, RungeKuttaSolver, TimeSeries, TimeParameters) over the
C-ABI. On the CPU the demo program must compile and link against libsv_b200.so; on the GPU
it runs a stage derivative, a trial timestep and whole steps, which must equal the oracle's
bit for bit."""
import json
import os
import subprocess

import numpy as np
import pytest

import mfcm_b200
from mfcm_b200 import synth, EDGE_XMAX, EDGE_YMIN
from tests.scenarios import same, forcing

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "mfcm_b200", "lib")


def build_demo(out_dir):
    mfcm_b200.load_library()  # the library must exist (built by mfcm_b200/build.py)
    exe = os.path.join(out_dir, "facade_demo")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "facade_demo.cpp"), "-L", LIBDIR, "-lsv_b200",
           f"-Wl,-rpath,{LIBDIR}", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_facade_compiles_and_links(tmp_path):
    exe = build_demo(str(tmp_path))
    assert os.path.exists(exe)


def test_facade_header_compiles_for_float_and_datum_options(tmp_path):
    src = tmp_path / "f32.cpp"
    src.write_text('#include "mfcm_b200.hpp"\n'
                   "using namespace mfcm_b200;\n"
                   "int main() {\n"
                   "  auto mesh = std::make_shared<Cartesian2DMesh>(8, 8, 1.0, 1.0);\n"
                   "  auto tp = std::make_shared<TimeParameters>();\n"
                   "  Options o; o.datum64 = true;\n"
                   "  using S = SaintVenantSolver<double, float>;\n"
                   "  try {\n"
                   "    RungeKuttaSolver<S> rk(tp, \"ralston4\", mesh, o);\n"
                   "    rk.solver().set_eddy_viscosity(SV_EDDY_SMAGORINSKY);\n"
                   "    rk.solver().set_source_order({SV_TERM_EDDY, SV_TERM_MANNING});\n"
                   "    rk.solver().set_field(FieldId::eddy_mu, std::vector<double>(64, 0.5));\n"
                   "  } catch (const std::runtime_error&) {}\n"
                   "  return TimeSeries({0.0, 10.0}, {0.0, 1.0}).at(5.0) == 0.5 ? 0 : 1;\n"
                   "}\n")
    r = subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-L",
                        LIBDIR, "-lsv_b200", f"-Wl,-rpath,{LIBDIR}", "-o", str(tmp_path / "f32")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_num_steps_and_time_series_match_the_python_mirror(tmp_path):
    """TimeParameters::num_steps and ts_linterp in the header agree with mfcm_b200's."""
    src = tmp_path / "ts.cpp"
    src.write_text('#include <cstdio>\n#include "mfcm_b200.hpp"\nusing namespace mfcm_b200;\n'
                   "int main() {\n"
                   "  TimeSeries ts({0.0, 600.0, 600.001, 3600.0}, {1.0, 1.0, 0.0, 0.0});\n"
                   "  double q[] = {0.0, 300.0, 600.0005, 5000.0};\n"
                   "  for (double t : q) std::printf(\"%.17g\\n\", ts.at(t));\n"
                   "  double ends[] = {3600.0, 3600.0000001, 3601.0};\n"
                   "  for (double e : ends) { TimeParameters p; p.end_time = e; std::printf(\"%zu\\n\", p.num_steps()); }\n"
                   "}\n")
    exe = tmp_path / "ts"
    r = subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    ts = mfcm_b200.TimeSeries([0.0, 600.0, 600.001, 3600.0], [1.0, 1.0, 0.0, 0.0])
    assert [float(x) for x in out[:4]] == [ts.at(t) for t in (0.0, 300.0, 600.0005, 5000.0)]
    assert [int(x) for x in out[4:]] == [mfcm_b200.num_steps(0.0, e, 60.0) for e in (3600.0, 3600.0000001, 3601.0)]


@pytest.mark.gpu
def test_facade_run_matches_the_oracle(tmp_path):
    from oracle.sv_oracle_py import OracleSolver
    nx, ny, dx, steps, L = 48, 40, 5.0, 3, 20.0
    rain = 60 * synth.MM_PER_H
    edges = EDGE_XMAX | EDGE_YMIN
    z = synth.plane_with_gaussians(nx, ny, dx, seed=9)
    h = np.full((ny, nx), 2e-3)
    z.astype(np.float64).tofile(tmp_path / "z.bin")
    h.astype(np.float64).tofile(tmp_path / "h.bin")
    exe = build_demo(str(tmp_path))
    r = subprocess.run([exe, str(tmp_path), str(nx), str(ny), repr(dx), str(steps), repr(L), repr(rain), str(edges)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert res["threw_on_bad_scheme"] is True

    o = OracleSolver(nx, ny, dx, cn_target=0.5, step_duration=L, rain_mode="physical")
    o.set_field("Z", z)
    o.set_field("H", h)
    o.set_field("U", np.zeros_like(h))
    o.set_field("V", np.zeros_like(h))
    o.set_manning(0.03, 0.03, 0.1, 0.3)
    o.set_forcing(forcing((rain, rain), head=(0.0, 0.0), edges=edges))
    o.eval_dudt(0, 0.0, 0.1)
    k0 = o.get_field("DHDT")
    cn, rep, nd = o.do_timestep(0.0, 0.1)
    per_step = []
    for i in range(steps):
        f = forcing((rain, rain), head=(0.0, 0.0), edges=edges)
        o.set_forcing(f)
        st = o.advance()  # this step's counts, like RungeKuttaSolver::step
        per_step.append([st["accepted"], st["repeated"]])
    assert same(np.fromfile(tmp_path / "k0_h.bin").reshape(ny, nx), k0)
    assert res["trial"] == [cn, int(rep), nd]
    assert res["steps"] == per_step
    for f in ("h", "u", "v"):
        assert same(np.fromfile(tmp_path / f"{f}.bin.out").reshape(ny, nx), o.get_field(f.upper())), f
    so = o.stats()
    assert res["volume"] == so["volume"] and res["dt"] == o.get_dt()
