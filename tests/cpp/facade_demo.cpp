// Drives the B200 library through the C++ facade (include/mfcm_b200.hpp) the way the
// reference's main loop drives RungeKuttaSolver<SaintVenantSolver<double, double,
// Cartesian2DMesh>> (src/mfcm.cpp:19-36): one stage derivative, one trial timestep, then
// whole steps through solve(). Inputs and outputs are raw float64 files so the test can
// compare every value with the oracle.
//
//   facade_demo <dir> <nx> <ny> <dx> <steps> <step seconds> <rain m/s> <head edges>
//   reads  <dir>/z.bin, <dir>/h.bin (nx*ny doubles each, row-major)
//   writes <dir>/k0_h.bin (dh/dt of U_[0]), <dir>/h.bin.out, u.bin.out, v.bin.out
//   prints one JSON line: the trial timestep and the per-step counts and tallies
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "mfcm_b200.hpp"

using namespace mfcm_b200;

static std::vector<double> read_bin(const std::string& path, std::size_t n) {
  std::vector<double> v(n);
  std::ifstream f(path, std::ios::binary);
  if (!f.read(reinterpret_cast<char*>(v.data()), std::streamsize(n * sizeof(double))))
    throw std::runtime_error("cannot read " + path);
  return v;
}

static void write_bin(const std::string& path, const std::vector<double>& v) {
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char*>(v.data()), std::streamsize(v.size() * sizeof(double)));
}

int main(int argc, char** argv) {
  if (argc != 9) {
    std::cerr << "usage: facade_demo dir nx ny dx steps step_seconds rain_m_s head_edges\n";
    return 2;
  }
  const std::string dir = argv[1];
  const uint64_t nx = std::strtoull(argv[2], nullptr, 10), ny = std::strtoull(argv[3], nullptr, 10);
  const double dx = std::atof(argv[4]);
  const int steps = std::atoi(argv[5]);
  const double L = std::atof(argv[6]), rain = std::atof(argv[7]);
  const unsigned edges = unsigned(std::atoi(argv[8]));
  try {
    // an unknown coefficient set is reported the reference's way: std::runtime_error
    bool threw = false;
    try {
      named_coefficient_set("no-such-scheme");
    } catch (const std::runtime_error&) {
      threw = true;
    }
    auto mesh = std::make_shared<Cartesian2DMesh>(nx, ny, dx, dx);
    auto tp = std::make_shared<TimeParameters>();
    tp->start_time = 0.0;
    tp->end_time = L * steps;
    tp->step_duration = L;
    tp->initial_timestep = 1.0;
    Options opt;
    opt.cn_target = 0.5;
    opt.physical_rain_clamp = true;
    using Solver = SaintVenantSolver<double, double, Cartesian2DMesh>;
    RungeKuttaSolver<Solver> rk(tp, "classic", mesh, opt);
    Solver& sv = rk.solver();
    const std::size_t n = mesh->cell_count();
    sv.set_field(FieldId::z_bed, read_bin(dir + "/z.bin", n));
    StateCopy s0{read_bin(dir + "/h.bin", n), std::vector<double>(n, 0.0), std::vector<double>(n, 0.0)};
    sv.set_state(s0);
    sv.set_manning(0.03, 0.03, 0.1, 0.3);
    TimeSeries rain_ts({0.0, 1e9}, {rain, rain});
    StepBoundaries b;
    b.rain_kind = StepBoundaries::Rain::uniform;
    b.rain = &rain_ts;
    b.head = edges != 0;
    b.head_edges = edges;
    sv.start_new_step(0.0, b);
    sv.update_dUdt(0, 0.0, 0.1);
    write_bin(dir + "/k0_h.bin", sv.dUdt(0).h);
    auto trial = rk.do_timestep(0.0, 0.1);
    auto res = rk.solve([&](double) { return b; });
    StateCopy out = sv.state(0);
    write_bin(dir + "/h.bin.out", out.h);
    write_bin(dir + "/u.bin.out", out.u);
    write_bin(dir + "/v.bin.out", out.v);
    sv_stats st = sv.end_of_step(tp->end_time);
    std::printf("{\"threw_on_bad_scheme\": %s, \"trial\": [%.17g, %d, %.17g], \"steps\": [", threw ? "true" : "false",
                trial.control_number, trial.repeat_timestep ? 1 : 0, trial.new_dt);
    for (std::size_t i = 0; i < res.size(); ++i)
      std::printf("%s[%zu, %zu]", i ? ", " : "", res[i].num_timesteps, res[i].num_repeated_timesteps);
    std::printf("], \"volume\": %.17g, \"rain_in\": %.17g, \"outflow\": %.17g, \"dt\": %.17g}\n", st.volume,
                st.rain_in, st.outflow, rk.current_timestep());
  } catch (const std::exception& e) {
    std::cerr << "error: " << e.what() << "\n";
    return 1;
  }
  return 0;
}
