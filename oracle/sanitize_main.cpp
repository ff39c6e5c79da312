// sanitize_main.cpp -- TEST INFRASTRUCTURE: drives the CPU oracle (sv_oracle_capi.cpp) through
// every entry point under AddressSanitizer and UndefinedBehaviorSanitizer.
//
// oracle/build.py compiles this file together with sv_oracle_capi.cpp into
// oracle/_build/sv_oracle_san (-fsanitize=address,undefined -fno-sanitize-recover=all), and
// tests/test_oracle_sanitize.py runs it. Any out-of-bounds access, use after free, leak,
// signed overflow, misaligned load or invalid shift in the oracle ends the run with a
// non-zero status and the sanitizer's report; a clean run prints "sanitized run ok" and the
// number of calls it made.
//
// The cases are the edges the parity tests reach: single cells, single rows and columns,
// ragged grids, coded-out (NaN) bed cells, every tableau, every rain and head kind, the
// eddy-viscosity modes, both source-term orders, both precisions, per-function evaluation
// with every field read back, and whole steps with and without the dt clamp.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "../include/sv.h"

extern "C" {
int svo_create(const sv_mesh_desc* mesh, const sv_params* params, void** out);
void svo_destroy(void* h);
int svo_set_field(void* h, int id, const double* src, uint64_t n);
int svo_get_field(void* h, int id, double* dst, uint64_t n);
int svo_set_manning(void* h, double a, double b, double c, double d);
int svo_set_eddy_viscosity(void* h, int mode, double mu, double mc, double ms);
int svo_set_source_order(void* h, const int* terms, int n);
int svo_set_forcing(void* h, const sv_forcing* f);
int svo_set_dt(void* h, double dt);
int svo_get_dt(void* h, double* dt);
int svo_eval_dudt(void* h, int state_no, double t_sub, double dt);
int svo_do_timestep(void* h, double t_local, double dt, double* cn, int* repeat, double* new_dt);
int svo_accept(void* h);
int svo_advance(void* h, sv_stats* out);
int svo_get_stats(void* h, sv_stats* out);
int svo_set_stats(void* h, const sv_stats* in);
double svo_pow43(double x);
double svo_minmod3(double ul, double dxl, double uc, double dxr, double ur);
const char* svo_last_error(void);
}

namespace {

uint64_t g_calls = 0;

// a small deterministic generator (64-bit LCG, top 53 bits) for the synthetic fields
struct Rng {
  uint64_t s;
  explicit Rng(uint64_t seed) : s(seed * 6364136223846793005ull + 1442695040888963407ull) {}
  double uniform() {
    s = s * 6364136223846793005ull + 1442695040888963407ull;
    return double(s >> 11) * (1.0 / 9007199254740992.0);
  }
  double range(double a, double b) { return a + (b - a) * uniform(); }
};

void check(int rc, const char* what) {
  ++g_calls;
  if (rc != 0) {
    std::fprintf(stderr, "%s failed (%d): %s\n", what, rc, svo_last_error());
    std::exit(2);
  }
}

struct Case {
  uint64_t nx, ny;
  double dx, dy;
  int precision;
  int rk;
  int nan_cells;
  int rain_kind;
  int head_kind;
  int eddy;
  int eloss_first;
};

void run_case(const Case& c, uint64_t seed) {
  sv_mesh_desc m{c.nx, c.ny, c.dx, c.dy, 0.0, 0.0};
  sv_params p{};
  p.precision = c.precision;
  p.rk_method = c.rk;
  p.cn_target = 0.5;
  p.step_duration = 2.0;
  p.initial_dt = 0.05;
  p.max_dt = (seed & 1) ? 0.5 : 0.0;
  p.rain_mode = int(seed % 2);
  p.manning = 1;
  p.head_first = int((seed >> 1) & 1);
  p.flags = c.eloss_first ? SV_FLAG_ELOSS_FIRST : 0;
  void* h = nullptr;
  check(svo_create(&m, &p, &h), "create");
  const uint64_t n = c.nx * c.ny;
  const uint64_t nf = (c.nx + 1) * c.ny + (c.ny + 1) * c.nx;
  Rng r(seed);
  std::vector<double> z(n), d(n), u(n), v(n), a(n), b(n);
  for (uint64_t i = 0; i < n; ++i) {
    const double x = double(i % c.nx) * c.dx, y = double(i / c.nx) * c.dy;
    z[i] = 0.01 * x + 0.005 * y + r.range(0.0, 0.3);
    d[i] = r.uniform() < 0.3 ? 0.0 : r.range(0.0, 0.5);
    u[i] = r.range(-0.5, 0.5);
    v[i] = r.range(-0.5, 0.5);
  }
  for (int k = 0; k < c.nan_cells && n > 1; ++k) z[uint64_t(r.uniform() * double(n)) % n] = NAN;
  check(svo_set_field(h, SV_FIELD_Z, z.data(), n), "set Z");
  check(svo_set_field(h, SV_FIELD_H, d.data(), n), "set H");
  check(svo_set_field(h, SV_FIELD_U, u.data(), n), "set U");
  check(svo_set_field(h, SV_FIELD_V, v.data(), n), "set V");
  check(svo_set_manning(h, 0.03, 0.05, 0.1, 0.3), "manning");
  for (uint64_t i = 0; i < n; ++i) a[i] = r.range(0.02, 0.06);
  check(svo_set_field(h, SV_FIELD_N_SHALLOW, a.data(), n), "set n_shallow");
  if (c.eddy) check(svo_set_eddy_viscosity(h, c.eddy, 0.5, 0.05, 0.5), "eddy");
  if (c.eloss_first) {
    for (uint64_t i = 0; i < n; ++i) a[i] = r.range(0.0, 0.1);
    check(svo_set_field(h, SV_FIELD_ELOSS_FX, a.data(), n), "set eloss fx");
    check(svo_set_field(h, SV_FIELD_ELOSS_FY, a.data(), n), "set eloss fy");
    const int order[3] = {2, 1, 3};
    check(svo_set_source_order(h, order, c.eddy ? 3 : 2), "source order");
  }
  if (seed % 3 == 0) {
    for (uint64_t i = 0; i < n; ++i) { a[i] = r.range(0.0, 2e-6); b[i] = r.range(0.0, 0.02); }
    check(svo_set_field(h, SV_FIELD_INFIL_RATE, a.data(), n), "set infiltration rate");
    check(svo_set_field(h, SV_FIELD_INFIL_CAP, b.data(), n), "set infiltration capacity");
  }
  sv_forcing f{};
  f.rain_kind = c.rain_kind;
  f.rain_q0 = 2e-5;
  f.rain_q1 = 1e-5;
  f.head_kind = c.head_kind;
  f.head_edges = SV_EDGE_XMIN | SV_EDGE_YMAX;
  f.head_h0 = 0.05;
  f.head_h1 = 0.1;
  check(svo_set_forcing(h, &f), "forcing");
  // per-cell boundary fields after the forcing (setting the forcing resets them)
  if (c.rain_kind == SV_RAIN_FIELDS) {
    for (uint64_t i = 0; i < n; ++i) { a[i] = r.range(0.0, 3e-5); b[i] = r.range(0.0, 3e-5); }
    check(svo_set_field(h, SV_FIELD_QBDY0, a.data(), n), "set qbdy0");
    check(svo_set_field(h, SV_FIELD_QBDY1, b.data(), n), "set qbdy1");
  }
  if (c.rain_kind == SV_RAIN_PATTERN) {
    for (uint64_t i = 0; i < n; ++i) a[i] = r.range(0.0, 2.0);
    check(svo_set_field(h, SV_FIELD_RAIN_PATTERN, a.data(), n), "set rain pattern");
  }
  if (c.head_kind == SV_HEAD_FIELDS || c.head_kind == SV_STAGE_FIELDS) {
    for (uint64_t i = 0; i < n; ++i) {
      a[i] = r.uniform() < 0.8 ? NAN : r.range(0.0, 0.2);
      b[i] = std::isnan(a[i]) ? NAN : a[i] + 0.01;
    }
    check(svo_set_field(h, SV_FIELD_HBDY0, a.data(), n), "set hbdy0");
    check(svo_set_field(h, SV_FIELD_HBDY1, b.data(), n), "set hbdy1");
  }
  // one evaluation of dU/dt with every cell and face field read back
  check(svo_eval_dudt(h, 0, 0.25, 0.05), "eval_dudt");
  std::vector<double> out(nf > n ? nf : n);
  const int cell_ids[] = {SV_FIELD_DHDT, SV_FIELD_DUDT, SV_FIELD_DVDT, SV_FIELD_DHDX, SV_FIELD_DUDX,
                          SV_FIELD_DVDX, SV_FIELD_DHDY, SV_FIELD_DUDY, SV_FIELD_DVDY, SV_FIELD_DZDX,
                          SV_FIELD_DZDY, SV_FIELD_Z, SV_FIELD_H, SV_FIELD_U, SV_FIELD_V};
  for (int id : cell_ids) check(svo_get_field(h, id, out.data(), n), "get cell field");
  const int face_ids[] = {SV_FIELD_FLUX_H, SV_FIELD_FLUX_U, SV_FIELD_FLUX_V, SV_FIELD_FLUX_Z,
                          SV_FIELD_FLUX_BRANCH};
  for (int id : face_ids) check(svo_get_field(h, id, out.data(), nf), "get face field");
  // one timestep by hand, with every stage's state and derivative read back
  double cn = 0.0, nd = 0.0;
  int rep = 0;
  check(svo_do_timestep(h, 0.0, 0.05, &cn, &rep, &nd), "do_timestep");
  const int stages[] = {1, 2, 2, 2, 3, 3, 3, 3, 3, 4, 4, 4};
  for (int s = 0; s <= stages[c.rk]; ++s)
    for (int k = 0; k < 3; ++k) check(svo_get_field(h, SV_FIELD_STATE_BASE + 3 * s + k, out.data(), n), "get stage");
  for (int s = 0; s < stages[c.rk]; ++s)
    for (int k = 0; k < 3; ++k) check(svo_get_field(h, SV_FIELD_K_BASE + 3 * s + k, out.data(), n), "get k");
  if (!rep) check(svo_accept(h), "accept");
  // a bounded run of timesteps on the rough state (its dt may collapse: the reference's
  // thin-film blow-up), then whole steps from a calm state (a 0.2 m lake at rest, which ends
  // its steps), a checkpoint round trip of the counters, and the dt accessors
  double t = 0.0, dt_now = nd;
  for (int k = 0; k < 8 && dt_now > 0.0 && std::isfinite(dt_now); ++k) {
    check(svo_do_timestep(h, t, dt_now, &cn, &rep, &nd), "do_timestep");
    if (!rep) {
      check(svo_accept(h), "accept");
      t += dt_now;
    }
    dt_now = nd;
  }
  for (uint64_t i = 0; i < n; ++i) { d[i] = 0.2; u[i] = 0.0; }
  check(svo_set_field(h, SV_FIELD_H, d.data(), n), "set H");
  check(svo_set_field(h, SV_FIELD_U, u.data(), n), "set U");
  check(svo_set_field(h, SV_FIELD_V, u.data(), n), "set V");
  sv_stats st{};
  check(svo_set_dt(h, 0.05), "set dt");
  for (int k = 0; k < 2; ++k) check(svo_advance(h, &st), "advance");
  check(svo_get_stats(h, &st), "stats");
  check(svo_set_stats(h, &st), "set stats");
  double dt = 0.0;
  check(svo_get_dt(h, &dt), "get dt");
  svo_destroy(h);
}

}  // namespace

int main() {
  const uint64_t shapes[][2] = {{1, 1}, {1, 9}, {9, 1}, {2, 2}, {23, 17}, {40, 3}, {3, 40}};
  const double spacing[][2] = {{3.0, 3.0}, {1.5, 1.5}, {1.5, 1.5}, {2.0, 5.0}, {3.0, 3.0}, {0.5, 0.25}, {4.0, 1.0}};
  uint64_t seed = 1;
  for (int precision : {SV_F64, SV_F32}) {
    for (int si = 0; si < 7; ++si) {
      for (int rk = 0; rk < 12; ++rk) {
        Case c{shapes[si][0], shapes[si][1], spacing[si][0], spacing[si][1], precision, rk,
               int(seed % 4) * 2, int(seed % 4), int(seed % 5), int(seed % 3), int(seed % 2)};
        run_case(c, seed++);
      }
    }
  }
  // the oracle's scalar helpers across their ranges, zero and non-finite arguments included
  volatile double sink = 0.0;
  const double xs[] = {0.0, 1e-300, 1e-8, 0.5, 1.0, 2.0, 1e8, INFINITY, NAN};
  for (double x : xs) sink = svo_pow43(x);
  for (double a : xs)
    for (double b : xs) sink = svo_minmod3(a, 1.0, b, 2.0, -a);
  (void)sink;
  std::printf("sanitized run ok: %llu calls\n", (unsigned long long)g_calls);
  return 0;
}
