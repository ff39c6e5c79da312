// sv_oracle.hpp -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
//
// CPU restatement of the reference's 2-D Saint-Venant explicit Runge-Kutta time step
// (oojimaflib/mfcm). It is the checker for the CUDA path: only tests/, the smoke check
// and bench.py's CPU-baseline leg may load it. The product library never links it.
//
// The reference cannot be compiled here (hipSYCL/AdaptiveCpp, Boost >= 1.78 and a clang
// front end are all absent), so this file restates its arithmetic, function by function,
// with the same pass structure (one loop per reference kernel, the same intermediate
// fields) and the same C++ type promotions (value type T, time type TT, mesh spacing as
// double). Each function names the reference lines it follows. Every loop over cells or
// faces is element-independent, so an OpenMP build gives results identical to a serial
// build; reductions are written to be order-independent (max) or fixed-order (sums).
//
// Parity status: the reference ships no tests, fixtures or golden vectors, and cannot be
// run here, so this restatement is pinned only by its own known-answer tests, by an
// independent numpy restatement of the same lines (oracle/sv_oracle_np.py) that must agree
// bit for bit, and by the committed fixtures under tests/golden/. Parity is "unpinned"
// against the reference binary itself.
//
// Documented choices where the reference is unspecified:
//  * sycl::sign/fmax/min/mix/smoothstep follow the SYCL 2020 / OpenCL C built-in
//    definitions (see the helpers below).
//  * sycl::pow(x, 4/3) is replaced by sv_math::pow43 (mfcm_b200/csrc/sv_pow43.h), shared
//    with the CUDA path, for T = double; for T = float std::pow is used.
//  * The control-number max reduction propagates NaN (the reference's sycl::maximum
//    result with a NaN operand depends on the combine order).
//  * ts_linterp reads past the end of the knot array when the time is at or beyond the
//    last knot (src/Input/TimeSeries.cpp:31-40); here it extrapolates the last segment.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../mfcm_b200/csrc/sv_pow43.h"

namespace svo {

// ---------------------------------------------------------------------------------------
// SYCL built-ins (SYCL 2020 section 4.17.5 "common functions" / OpenCL C 6.15.4).
// ---------------------------------------------------------------------------------------
// sign(x): 1.0 if x > 0, -1.0 if x < 0, +-0.0 for +-0.0, 0.0 for NaN.
template <typename T> inline T ssign(T x) {
  if (x > T(0)) return T(1);
  if (x < T(0)) return T(-1);
  if (x == x) return x;
  return T(0);
}
// min(x, y): "returns y if y < x, otherwise x".
template <typename T> inline T smin(T x, T y) { return (y < x) ? y : x; }
// fmax: IEEE maxNum (the non-NaN operand when exactly one is NaN).
template <typename T> inline T sfmax(T x, T y) { return std::fmax(x, y); }
// mix(x, y, a) = x + (y - x) * a
template <typename T> inline T smix(T x, T y, T a) { return x + (y - x) * a; }
// clamp(x, lo, hi) = fmin(fmax(x, lo), hi)
template <typename T> inline T sclamp(T x, T lo, T hi) { return std::fmin(std::fmax(x, lo), hi); }
// smoothstep(e0, e1, x): t = clamp((x - e0) / (e1 - e0), 0, 1); t * t * (3 - 2 * t)
template <typename T> inline T ssmoothstep(T e0, T e1, T x) {
  T t = sclamp((x - e0) / (e1 - e0), T(0), T(1));
  return t * t * (T(3) - T(2) * t);
}
template <typename T> inline T spow43(T x);
template <> inline double spow43<double>(double x) { return sv_math::pow43(x); }
template <> inline float spow43<float>(float x) { return std::pow(x, float(4.0) / float(3.0)); }

// ---------------------------------------------------------------------------------------
// Cartesian2DMesh / Cartesian2DMeshAccessor (src/Mesh/Cartesian2DMesh.hpp:28-521),
// rotation angle 0: dx = |cell width|, dy = |cell height| (Cartesian2DMesh.cpp:41-55).
// ---------------------------------------------------------------------------------------
struct Mesh {
  size_t nx = 0, ny = 0;
  double dx = 1.0, dy = 1.0;
  size_t ncells() const { return nx * ny; }                       // :92-96
  size_t nfaces() const { return (nx + 1) * ny + (ny + 1) * nx; }  // :98-103
  double cell_area() const { return dx * dy; }                     // :296-299

  struct Adj { size_t lhs, rhs; int edge, dir; double d; };
  // get_adjacent_cells (:379-435): vertical faces first, then horizontal faces.
  Adj adjacent_cells(size_t f) const {
    Adj a{};
    if (f < (nx + 1) * ny) {
      a.dir = 0; a.d = dx;
      size_t fx = f % (nx + 1), fy = f / (nx + 1);
      if (fx < nx) {
        a.rhs = fy * nx + fx;
        if (fx > 0) { a.edge = 0; a.lhs = fy * nx + (fx - 1); }
        else { a.edge = -1; a.lhs = a.rhs; }
      } else {
        a.lhs = fy * nx + (fx - 1); a.rhs = a.lhs; a.edge = 1;
      }
    } else {
      a.dir = 1; a.d = dy;
      size_t f2 = f - (nx + 1) * ny;
      size_t fx = f2 % nx, fy = f2 / nx;
      if (fy < ny) {
        a.rhs = fy * nx + fx;
        if (fy > 0) { a.edge = 0; a.lhs = (fy - 1) * nx + fx; }
        else { a.edge = -1; a.lhs = a.rhs; }
      } else {
        a.lhs = (fy - 1) * nx + fx; a.rhs = a.lhs; a.edge = 1;
      }
    }
    return a;
  }
  struct Faces { size_t w, e; double dx; size_t s, n; double dy; };
  // get_adjacent_faces (:447-460)
  Faces adjacent_faces(size_t c) const {
    size_t cx = c % nx, cy = c / nx;
    Faces r;
    r.w = cy * (nx + 1) + cx; r.e = r.w + 1; r.dx = dx;
    r.s = (nx + 1) * ny + cy * nx + cx; r.n = r.s + nx; r.dy = dy;
    return r;
  }
  struct Off { size_t i; double d; };
  // get_object_{west,east,north,south}<Cell> (:477-519)
  Off west(size_t i) const { return (i % nx > 0) ? Off{i - 1, dx} : Off{i, 0.0}; }
  Off east(size_t i) const { return (i % nx < nx - 1) ? Off{i + 1, dx} : Off{i, 0.0}; }
  Off north(size_t i) const { return (i / nx < ny - 1) ? Off{i + nx, dy} : Off{i, 0.0}; }
  Off south(size_t i) const { return (i / nx > 0) ? Off{i - nx, dy} : Off{i, 0.0}; }
};

// ---------------------------------------------------------------------------------------
// Minmod3 with theta = 2 (src/SpatialDerivative/Minmod3.hpp:22-84).
// ---------------------------------------------------------------------------------------
template <typename T>
inline T minmod3(const T& Ul, const double& dxl, const T& Uc, const double& dxr, const T& Ur) {
  const T theta = 2.0;
  T lhs = std::numeric_limits<T>::quiet_NaN();
  if (dxl > 0.01 * dxr) lhs = theta * (Uc - Ul) / T(dxl);
  T rhs = std::numeric_limits<T>::quiet_NaN();
  if (dxr > 0.01 * dxl) rhs = theta * (Ur - Uc) / T(dxr);
  T central = 0.0;
  T total_dx = dxl + dxr;
  if (total_dx > 1e-6) central = (Ur - Ul) / T(dxl + dxr);
  T outer = std::numeric_limits<T>::quiet_NaN();
  if (std::isnan(lhs)) outer = rhs;
  else if (std::isnan(rhs)) outer = lhs;
  else outer = T(0.5) * (ssign(lhs) + ssign(rhs)) * smin(std::fabs(lhs), std::fabs(rhs));
  if (std::isnan(outer)) return central;
  return T(0.5) * (ssign(outer) + ssign(central)) * smin(std::fabs(outer), std::fabs(central));
}

// SpatialDerivativeOperationKernel (src/SpatialDerivative/SpatialDerivative.hpp:190-208):
// X uses (west, east); Y uses (north, south) as (left, right), i.e. dU/dy = -dU/drow.
template <typename T>
inline void slope_x(const Mesh& m, const T* s, T* d, size_t i) {
  auto l = m.west(i); auto r = m.east(i);
  d[i] = minmod3<T>(s[l.i], l.d, s[i], r.d, s[r.i]);
}
template <typename T>
inline void slope_y(const Mesh& m, const T* s, T* d, size_t i) {
  auto l = m.north(i); auto r = m.south(i);
  d[i] = minmod3<T>(s[l.i], l.d, s[i], r.d, s[r.i]);
}

// ---------------------------------------------------------------------------------------
// Runge-Kutta tableaux (src/TemporalScheme/RungeKutta.cpp:21-115). Row i of `a` holds
// c_i followed by a_{i,1..i-1}; the last row holds 0 followed by b_1..b_N.
// ---------------------------------------------------------------------------------------
struct Tableau {
  std::vector<std::vector<double>> a;
  size_t nsteps() const { return a.size() - 1; }
  double A(size_t i, size_t j) const { return a[i - 1][j]; }  // RungeKutta.hpp:102-105
  double b(size_t i) const { return a[a.size() - 1][i]; }     // :110-113
  double c(size_t i) const { return a[i - 1][0]; }            // :118-121
};

inline const char* const kTableauNames[] = {"euler", "midpoint", "heun2", "ralston2", "kutta3", "heun3",
                                            "wray3", "ralston3", "ssprk3", "classic", "ralston4", "3/8rule"};
inline Tableau named_tableau(int id) {
  switch (id) {
    case 0: return {{{0.0}, {0.0, 1.0}}};
    case 1: return {{{0.0}, {0.5, 0.5}, {0.0, 0.0, 1.0}}};
    case 2: return {{{0.0}, {1.0, 1.0}, {0.0, 0.5, 0.5}}};
    case 3: return {{{0.0}, {2.0 / 3.0, 2.0 / 3.0}, {0.0, 0.25, 0.75}}};
    case 4: return {{{0.0}, {0.5, 0.5}, {1.0, -1.0, 2.0}, {0.0, 1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0}}};
    case 5: return {{{0.0}, {1.0 / 3.0, 1.0 / 3.0}, {2.0 / 3.0, 0.0, 2.0 / 3.0}, {0.0, 0.25, 0.0, 0.75}}};
    case 6: return {{{0.0}, {8.0 / 15.0, 8.0 / 15.0}, {2.0 / 3.0, 0.25, 5.0 / 12.0}, {0.0, 0.25, 0.0, 0.75}}};
    case 7: return {{{0.0}, {0.5, 0.5}, {0.75, 0.0, 0.75}, {0.0, 2.0 / 9.0, 1.0 / 3.0, 4.0 / 9.0}}};
    case 8: return {{{0.0}, {1.0, 1.0}, {0.5, 0.25, 0.25}, {0.0, 1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0}}};
    case 9: return {{{0.0}, {0.5, 0.5}, {0.5, 0.0, 0.5}, {1.0, 0.0, 0.0, 1.0},
                     {0.0, (1.0 / 6.0), (1.0 / 3.0), (1.0 / 3.0), (1.0 / 6.0)}}};
    case 10: return {{{0.0}, {0.4, 0.4}, {0.45573725, 0.29697761, 0.15875964},
                      {1.0, 0.21810040, -3.05096516, 3.83286476},
                      {0.0, 0.17476028, -0.55148066, 1.20553560, 0.17118478}}};
    case 11: return {{{0.0}, {1.0 / 3.0, 1.0 / 3.0}, {2.0 / 3.0, -1.0 / 3.0, 1.0}, {1.0, 1.0, -1.0, 1.0},
                      {0.0, 1.0 / 8.0, 3.0 / 8.0, 3.0 / 8.0, 1.0 / 8.0}}};
  }
  throw std::runtime_error("Unknown name for Runge Kutta scheme.");
}

// Time series with linear interpolation (ts_linterp, src/Input/TimeSeries.cpp:26-47).
template <typename TT, typename T>
inline T ts_linterp(const std::vector<TT>& t, const std::vector<T>& v, const TT& time) {
  size_t i1 = 1;
  for (; i1 < t.size(); ++i1)
    if (t[i1] > time) break;
  if (i1 >= t.size()) i1 = t.size() - 1;  // past the last knot: extrapolate (reference UB)
  size_t i0 = i1 - 1;
  TT t0 = t[i0], t1 = t[i1];
  T v0 = v[i0], v1 = v[i1];
  TT dvdt = (v1 - v0) / (t1 - t0);
  TT dt = time - t0;
  T result = v0 + dvdt * dt;
  return result;
}

// ---------------------------------------------------------------------------------------
// Problem description shared with the C-ABI (see oracle/sv_oracle_capi.cpp).
// ---------------------------------------------------------------------------------------
struct Params {
  int rk_method = 9;          // classic
  double cn_target = 1.0;     // RungeKutta.cpp:154
  double step_duration = 60;  // TimeParameters.cpp:29-32
  double initial_dt = 1.0;    // TimeParameters.cpp:34
  double max_dt = 0.0;        // 0 = off (the reference never clamps)
  int rain_mode = 0;          // 0 = reference clamp, 1 = physical (sign-corrected) clamp
  int manning = 1;            // Manning source term present
  int head_first = 0;         // boundary order: 0 = discharge then head, 1 = head then discharge
  int eloss_first = 0;        // source order: 1 = energy loss listed before Manning roughness
  // EddyViscositySourceTerm (EddyViscositySourceTerm.cpp:112-137): 0 off, 1 constant
  // coefficient (the F_EDDY_MU field when set, else eddy_mu), 2 Smagorinsky
  int eddy = 0;
  double eddy_mu = 1.0, eddy_c = 0.05, eddy_s = 0.5;
  // the momentum terms in configuration order (1 roughness, 2 energy loss, 3 eddy viscosity);
  // when not set, roughness and energy loss per eloss_first, then eddy viscosity
  int term_order[3] = {1, 2, 3};
  int order_set = 0;
};

enum Field : int {
  F_Z = 0, F_H = 1, F_U = 2, F_V = 3, F_N_SHALLOW = 4, F_N_DEEP = 5, F_D_SHALLOW = 6, F_D_DEEP = 7,
  F_QBDY0 = 8, F_QBDY1 = 9, F_HBDY0 = 10, F_HBDY1 = 11, F_RAIN_PATTERN = 12,
  F_INFIL_RATE = 13, F_INFIL_CAP = 14, F_ELOSS_FX = 15, F_ELOSS_FY = 16, F_EDDY_MU = 18,
  F_DHDT = 20, F_DUDT = 21, F_DVDT = 22, F_DHDX = 23, F_DUDX = 24, F_DVDX = 25,
  F_DHDY = 26, F_DUDY = 27, F_DVDY = 28, F_DZDX = 29, F_DZDY = 30, F_NH = 31, F_SF = 32,
  F_FLUX_H = 40, F_FLUX_U = 41, F_FLUX_V = 42, F_FLUX_Z = 43, F_FLUX_BRANCH = 44,
};

struct Forcing {
  // discharge (rainfall): 0 none, 1 uniform (q0, q1) on every cell, 2 per-cell fields
  // QBDY0/QBDY1, 3 per-cell pattern P times (q0, q1)
  int rain_kind = 0;
  double rain_q0 = 0, rain_q1 = 0;
  // head (outflow): 0 none, 1 one-cell strips along the edges in head_edges with scalar
  // targets (h0, h1), 2 per-cell fields HBDY0/HBDY1 (NaN = not selected)
  int head_kind = 0;
  unsigned head_edges = 0;  // bit0 x=0, bit1 x=nx-1, bit2 y=0, bit3 y=ny-1
  double head_h0 = 0, head_h1 = 0;
};

struct Stats {
  uint64_t accepted = 0, repeated = 0;
  double volume = 0, rain_in = 0, outflow = 0, wall_in = 0;
};

// Fixed-order compensated (Neumaier) sum: deterministic and accurate to ~1 ulp of the
// exact sum, so it serves as the reference value for the GPU's tree reductions.
inline double neumaier_sum(const double* x, size_t n) {
  double s = 0.0, c = 0.0;
  for (size_t i = 0; i < n; ++i) {
    double t = s + x[i];
    if (std::fabs(s) >= std::fabs(x[i])) c += (s - t) + x[i];
    else c += (x[i] - t) + s;
    s = t;
  }
  return s + c;
}

// ---------------------------------------------------------------------------------------
// SaintVenantSolver + RungeKuttaSolver + TypedTemporalScheme restated together.
// ---------------------------------------------------------------------------------------
class SolverBase {
 public:
  virtual ~SolverBase() {}
  virtual void set_field(int id, const double* src, size_t n) = 0;
  virtual void get_field(int id, double* dst, size_t n) const = 0;
  virtual void set_manning(double ns, double nd, double ds, double dd) = 0;
  virtual void set_eddy(int mode, double mu, double mc, double ms) = 0;
  virtual void set_source_order(const int* terms, int n) = 0;
  virtual void set_forcing(const Forcing& f) = 0;
  virtual void set_dt(double dt) = 0;
  virtual double get_dt() const = 0;
  virtual void update_dUdt(size_t state_no, double t_sub, double dt) = 0;
  virtual void do_timestep(double t_local, double dt, double* cn, int* repeat, double* new_dt) = 0;
  virtual void accept() = 0;
  virtual void step(Stats* st) = 0;
  virtual double volume() const = 0;
  virtual Stats stats() const = 0;
  virtual void set_stats(const Stats& s) = 0;
  virtual size_t state_count() const = 0;
  virtual void set_track_tallies(bool on) = 0;
};

template <typename TT, typename T>
class Solver final : public SolverBase {
  using Vec = std::vector<T>;
  struct State { Vec h, u, v; };

 public:
  Mesh m;
  Params p;
  Tableau tab;
  Vec z, dzdx, dzdy;                    // SaintVenantConstants (Constants.cpp:25-44)
  std::vector<State> U, K;              // U_[0..N], dUdt_[0..N-1] (Solver.cpp:44-50)
  State dUdx, dUdy;                     // Solver.cpp:57-58
  Vec fh, fu, fv, fz, fb;               // SaintVenantFluxes (Fluxes.cpp:24-42)
  Vec ns, nd, ds, dd, nh, Sf;           // ManningRoughnessSourceTerm (ManningRoughnessSourceTerm.hpp:111-117)
  Vec qb0, qb1, hb0, hb1, pattern;      // boundary xbdy0/xbdy1 (BoundarySourceTerm.hpp:44-45)
  Vec irate, icap;                      // InfiltrationSourceTerm (InfiltrationSourceTerm.hpp:106-109)
  Vec efx, efy;                         // EnergyLossSourceTerm (EnergyLossSourceTerm.hpp:199-202)
  unsigned present = 0;                 // which of those four fields were set (bits 0-3)
  Vec emu;                              // eddy viscosity coefficient field "mu"
  bool emu_set = false;
  Vec d2udx2, d2udy2, d2vdx2, d2vdy2;   // EddyViscositySourceTerm.hpp:154-157
  Forcing forcing;
  TT dt_;
  Stats st_;
  // tallies of the last evaluated stages, per state_no: sum over cells of the rain term
  // and of the head-boundary removal (k before head assignment minus k after)
  std::vector<double> rain_sum_, out_sum_, wall_sum_;
  bool track_tallies = true;  // off for the timed CPU baseline (the reference keeps no tallies)

  Solver(const Mesh& mesh, const Params& prm) : m(mesh), p(prm), tab(named_tableau(prm.rk_method)) {
    size_t n = m.ncells(), nf = m.nfaces(), N = tab.nsteps();
    z.assign(n, T(0)); dzdx.assign(n, T(0)); dzdy.assign(n, T(0));
    U.resize(N + 1); K.resize(N);
    for (auto& s : U) { s.h.assign(n, T(0)); s.u.assign(n, T(0)); s.v.assign(n, T(0)); }
    for (auto& s : K) { s.h.assign(n, T(0)); s.u.assign(n, T(0)); s.v.assign(n, T(0)); }
    for (State* s : {&dUdx, &dUdy}) { s->h.assign(n, T(0)); s->u.assign(n, T(0)); s->v.assign(n, T(0)); }
    fh.assign(nf, T(0)); fu.assign(nf, T(0)); fv.assign(nf, T(0)); fz.assign(nf, T(0)); fb.assign(nf, T(0));
    // ManningRoughnessSourceTerm::create_source_term defaults (ManningRoughnessSourceTerm.cpp:99-102)
    ns.assign(n, T(0.03)); nd.assign(n, T(0.3)); ds.assign(n, T(0.1)); dd.assign(n, T(0.3));
    nh.assign(n, T(0)); Sf.assign(n, T(0));
    qb0.assign(n, T(0)); qb1.assign(n, T(0));
    hb0.assign(n, std::numeric_limits<T>::quiet_NaN()); hb1.assign(n, std::numeric_limits<T>::quiet_NaN());
    pattern.assign(n, T(0));
    irate.assign(n, T(0)); icap.assign(n, T(0)); efx.assign(n, T(0)); efy.assign(n, T(0));
    emu.assign(n, T(0));
    for (Vec* d : {&d2udx2, &d2udy2, &d2vdx2, &d2vdy2}) d->assign(n, T(0));
    dt_ = TT(p.initial_dt);
    rain_sum_.assign(N, 0.0); out_sum_.assign(N, 0.0); wall_sum_.assign(N, 0.0);
    update_constants();
  }

  size_t state_count() const override { return U.size(); }
  void set_track_tallies(bool on) override { track_tallies = on; }

  void update_constants() {
    size_t n = m.ncells();
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; ++i) slope_x<T>(m, z.data(), dzdx.data(), i);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; ++i) slope_y<T>(m, z.data(), dzdy.data(), i);
  }

  Vec* field_ptr(int id) {
    switch (id) {
      case F_Z: return &z; case F_H: return &U[0].h; case F_U: return &U[0].u; case F_V: return &U[0].v;
      case F_N_SHALLOW: return &ns; case F_N_DEEP: return &nd; case F_D_SHALLOW: return &ds;
      case F_D_DEEP: return &dd; case F_QBDY0: return &qb0; case F_QBDY1: return &qb1;
      case F_HBDY0: return &hb0; case F_HBDY1: return &hb1; case F_RAIN_PATTERN: return &pattern;
      case F_INFIL_RATE: return &irate; case F_INFIL_CAP: return &icap;
      case F_ELOSS_FX: return &efx; case F_ELOSS_FY: return &efy; case F_EDDY_MU: return &emu;
      case F_DHDT: return &K[0].h; case F_DUDT: return &K[0].u; case F_DVDT: return &K[0].v;
      case F_DHDX: return &dUdx.h; case F_DUDX: return &dUdx.u; case F_DVDX: return &dUdx.v;
      case F_DHDY: return &dUdy.h; case F_DUDY: return &dUdy.u; case F_DVDY: return &dUdy.v;
      case F_DZDX: return &dzdx; case F_DZDY: return &dzdy; case F_NH: return &nh; case F_SF: return &Sf;
      case F_FLUX_H: return &fh; case F_FLUX_U: return &fu; case F_FLUX_V: return &fv;
      case F_FLUX_Z: return &fz; case F_FLUX_BRANCH: return &fb;
    }
    if (id >= 100 && id < 100 + 3 * (int)U.size()) {
      State& s = U[(id - 100) / 3];
      int c = (id - 100) % 3;
      return c == 0 ? &s.h : (c == 1 ? &s.u : &s.v);
    }
    if (id >= 200 && id < 200 + 3 * (int)K.size()) {
      State& s = K[(id - 200) / 3];
      int c = (id - 200) % 3;
      return c == 0 ? &s.h : (c == 1 ? &s.u : &s.v);
    }
    throw std::runtime_error("unknown field id");
  }
  const Vec* field_ptr(int id) const { return const_cast<Solver*>(this)->field_ptr(id); }

  void set_field(int id, const double* src, size_t n) override {
    Vec* f = field_ptr(id);
    if (n != f->size()) throw std::runtime_error("field size mismatch");
    for (size_t i = 0; i < n; ++i) (*f)[i] = T(src[i]);
    if (id == F_Z) update_constants();
    if (id >= F_INFIL_RATE && id <= F_ELOSS_FY) present |= 1u << (id - F_INFIL_RATE);
    if (id == F_EDDY_MU) emu_set = true;
  }
  void get_field(int id, double* dst, size_t n) const override {
    const Vec* f = field_ptr(id);
    if (n != f->size()) throw std::runtime_error("field size mismatch");
    for (size_t i = 0; i < n; ++i) dst[i] = double((*f)[i]);
  }
  void set_manning(double a, double b, double c, double d) override {
    std::fill(ns.begin(), ns.end(), T(a)); std::fill(nd.begin(), nd.end(), T(b));
    std::fill(ds.begin(), ds.end(), T(c)); std::fill(dd.begin(), dd.end(), T(d));
  }
  void set_eddy(int mode, double mu, double mc, double ms) override {
    if (mode < 0 || mode > 2) throw std::runtime_error("unknown eddy viscosity mode");
    p.eddy = mode; p.eddy_mu = mu; p.eddy_c = mc; p.eddy_s = ms;
  }
  void set_source_order(const int* terms, int n) override {
    if (n < 0 || n > 3) throw std::runtime_error("at most three source terms");
    bool seen[4] = {};
    int k = 0;
    for (int i = 0; i < n; ++i) {
      if (terms[i] < 1 || terms[i] > 3 || seen[terms[i]]) throw std::runtime_error("bad source order");
      seen[terms[i]] = true;
      p.term_order[k++] = terms[i];
    }
    for (int x = 1; x <= 3; ++x)
      if (!seen[x]) p.term_order[k++] = x;
    p.order_set = 1;
  }
  void set_dt(double dt) override { dt_ = TT(dt); }
  double get_dt() const override { return double(dt_); }
  Stats stats() const override { Stats s = st_; s.volume = volume(); return s; }
  void set_stats(const Stats& s) override {
    st_.accepted = s.accepted; st_.repeated = s.repeated; st_.rain_in = s.rain_in; st_.outflow = s.outflow;
    st_.wall_in = s.wall_in;
  }

  // start_new_step for the discharge and head boundaries
  // (DischargeBoundarySourceTerm.hpp:114-146, HeadBoundarySourceTerm.hpp:114-146): clear,
  // then add (discharge) or set (head) the values for [t, t + L] on the selection.
  // clear_values() is `x *= 0; x += 0` (Field.cpp:91-96), so NaN head targets outside the
  // selection stay NaN.
  void set_forcing(const Forcing& f) override {
    forcing = f;
    size_t n = m.ncells();
    for (size_t i = 0; i < n; ++i) { qb0[i] = qb0[i] * T(0.0) + T(0.0); qb1[i] = qb1[i] * T(0.0) + T(0.0); }
    if (f.rain_kind == 1) {
      T a = T(f.rain_q0), b = T(f.rain_q1);
      for (size_t i = 0; i < n; ++i) { qb0[i] += a; qb1[i] += b; }
    } else if (f.rain_kind == 3) {
      T a = T(f.rain_q0), b = T(f.rain_q1);
      for (size_t i = 0; i < n; ++i) { qb0[i] += pattern[i] * a; qb1[i] += pattern[i] * b; }
    }
    // rain_kind == 2: the caller uploads QBDY0/QBDY1 after this call
    // head_kind 3 is a stage boundary on edge strips (StageBoundarySourceTerm): the same
    // selection and values, read as water levels by stage_cell
    if (f.head_kind == 1 || f.head_kind == 3) {
      for (size_t i = 0; i < n; ++i) { hb0[i] = hb0[i] * T(0.0) + T(0.0); hb1[i] = hb1[i] * T(0.0) + T(0.0); }
      T a = T(f.head_h0), b = T(f.head_h1);
      for (size_t i = 0; i < n; ++i) {
        size_t x = i % m.nx, y = i / m.nx;
        bool sel = ((f.head_edges & 1u) && x == 0) || ((f.head_edges & 2u) && x == m.nx - 1) ||
                   ((f.head_edges & 4u) && y == 0) || ((f.head_edges & 8u) && y == m.ny - 1);
        if (sel) { hb0[i] = a; hb1[i] = b; }
      }
    } else if (f.head_kind == 0) {
      for (size_t i = 0; i < n; ++i) { hb0[i] = std::numeric_limits<T>::quiet_NaN(); hb1[i] = hb0[i]; }
    }
  }

  // SaintVenantFluxKernel::operator() (src/SaintVenant/FluxKernel.cpp:62-295)
  void flux_face(size_t fid, const State& S) {
    auto adj = m.adjacent_cells(fid);
    size_t lhs_id = adj.lhs, rhs_id = adj.rhs;
    int edge = adj.edge, dir = adj.dir;
    double dx = adj.d;
    T xdir = 1.0 - T(dir);
    T ydir = T(dir);
    T zb_L = z[lhs_id];
    T zb_R = z[rhs_id];
    auto zero = [&]() { fh[fid] = T(0.0); fu[fid] = T(0.0); fv[fid] = T(0.0); fz[fid] = T(0.0); fb[fid] = T(0.0); };
    if (zb_L != zb_L) {
      lhs_id = rhs_id;
      if (edge == 1) { zero(); return; }
      edge = -1;
    }
    if (zb_R != zb_R) {
      if (edge == -1) { zero(); return; }
      rhs_id = lhs_id;
      edge = 1;
    }
    T h_L = S.h[lhs_id] * (edge < 0 ? 0 : 1);
    T h_R = S.h[rhs_id] * (edge > 0 ? 0 : 1);
    T u_L = S.u[lhs_id] * (edge < 0 && xdir == 1 ? 0 : 1);
    T u_R = S.u[rhs_id] * (edge > 0 && xdir == 1 ? 0 : 1);
    T v_L = S.v[lhs_id] * (edge < 0 && ydir == 1 ? 0 : 1);
    T v_R = S.v[rhs_id] * (edge > 0 && ydir == 1 ? 0 : 1);
    T dhdx_L = dUdx.h[lhs_id] * (edge < 0 ? 0 : 1);
    T dhdx_R = dUdx.h[rhs_id] * (edge > 0 ? 0 : 1);
    T dhdy_L = dUdy.h[lhs_id] * (edge < 0 ? 0 : 1);
    T dhdy_R = dUdy.h[rhs_id] * (edge > 0 ? 0 : 1);
    T dudx_L = dUdx.u[lhs_id] * (edge < 0 && xdir == 1 ? 0 : 1);
    T dudx_R = dUdx.u[rhs_id] * (edge > 0 && xdir == 1 ? 0 : 1);
    T dudy_L = dUdy.u[lhs_id] * (edge < 0 && xdir == 1 ? 0 : 1);
    T dudy_R = dUdy.u[rhs_id] * (edge > 0 && xdir == 1 ? 0 : 1);
    T dvdx_L = dUdx.v[lhs_id] * (edge < 0 && ydir == 1 ? 0 : 1);
    T dvdx_R = dUdx.v[rhs_id] * (edge > 0 && ydir == 1 ? 0 : 1);
    T dvdy_L = dUdy.v[lhs_id] * (edge < 0 && ydir == 1 ? 0 : 1);
    T dvdy_R = dUdy.v[rhs_id] * (edge > 0 && ydir == 1 ? 0 : 1);
    T dzbdx_L = dzdx[lhs_id] * (edge < 0 ? 0 : 1);
    T dzbdx_R = dzdx[rhs_id] * (edge > 0 ? 0 : 1);
    T dzbdy_L = dzdy[lhs_id] * (edge < 0 ? 0 : 1);
    T dzbdy_R = dzdy[rhs_id] * (edge > 0 ? 0 : 1);
    if (edge < 0) zb_L = zb_R + h_R * 2.0f;
    if (edge > 0) zb_R = zb_L + h_L * 2.0f;
    T zb_m = zb_L + T(0.5) * dx * dzbdx_L * xdir + T(0.5) * dx * dzbdy_L * ydir;
    T h_m = h_L + T(0.5) * dx * dhdx_L * xdir + T(0.5) * dx * dhdy_L * ydir;
    T u_m = u_L + T(0.5) * dx * dudx_L * xdir + T(0.5) * dx * dudy_L * ydir;
    T v_m = v_L + T(0.5) * dx * dvdx_L * xdir + T(0.5) * dx * dvdy_L * ydir;
    T zb_p = zb_R + T(-0.5) * dx * dzbdx_R * xdir + T(-0.5) * dx * dzbdy_R * ydir;
    T h_p = h_R + T(-0.5) * dx * dhdx_R * xdir + T(-0.5) * dx * dhdy_R * ydir;
    T u_p = u_R + T(-0.5) * dx * dudx_R * xdir + T(-0.5) * dx * dudy_R * ydir;
    T v_p = v_R + T(-0.5) * dx * dvdx_R * xdir + T(-0.5) * dx * dvdy_R * ydir;
    T zb_f = sfmax(zb_m, zb_p);
    T y_m = zb_m + h_m;
    T y_p = zb_p + h_p;
    h_m = sfmax(h_m, T(0.0));
    h_p = sfmax(h_p, T(0.0));
    T c_m = std::sqrt(T(9.81) * h_m);
    T c_p = std::sqrt(T(9.81) * h_p);
    T branch = 5;
    if (y_m > zb_f && y_p > zb_f) {
      branch = 1;
      T spd_m = u_m * xdir + v_m * ydir;
      T spd_p = u_p * xdir + v_p * ydir;
      T hf_m = h_m * spd_m;
      T hf_p = h_p * spd_p;
      T uf_m = u_m * (T(1.0 - 0.5 * xdir) * spd_m) + T(9.81) * h_m * xdir;
      T uf_p = u_p * (T(1.0 - 0.5 * xdir) * spd_p) - T(9.81) * h_p * xdir;
      T vf_m = v_m * (T(1.0 - 0.5 * ydir) * spd_m) + T(9.81) * h_m * ydir;
      T vf_p = v_p * (T(1.0 - 0.5 * ydir) * spd_p) - T(9.81) * h_p * ydir;
      T a = sfmax(std::fabs(spd_p + ssign(spd_p) * c_p), std::fabs(spd_m + ssign(spd_m) * c_m));
      fh[fid] = T(0.5) * (hf_p + hf_m) - T(0.5) * a * (h_p - h_m);
      fu[fid] = T(0.5) * (uf_p + uf_m) - T(0.5) * a * (u_p - u_m);
      fv[fid] = T(0.5) * (vf_p + vf_m) - T(0.5) * a * (v_p - v_m);
      fz[fid] = (zb_m - zb_p) * T(9.81);
    } else if (y_m <= zb_f && y_p <= zb_f) {
      branch = 2;
      fh[fid] = T(0.0);
      if (zb_p > zb_m) {
        branch += 0.25;
        T uf_m = T(9.81) * h_m * xdir;
        T vf_m = T(9.81) * h_m * ydir;
        fu[fid] = T(0.5) * uf_m;
        fv[fid] = T(0.5) * vf_m;
        fz[fid] = -h_m * T(0.5) * T(9.81);
      } else {
        branch += 0.75;
        T uf_p = T(9.81) * h_p * xdir;
        T vf_p = T(9.81) * h_p * ydir;
        fu[fid] = T(-0.5) * uf_p;
        fv[fid] = T(-0.5) * vf_p;
        fz[fid] = h_p * T(0.5) * T(9.81);
      }
    } else if (y_m > zb_f) {
      branch = 3;
      T spd_m = u_m * xdir + v_m * ydir;
      T hf_m = h_m * spd_m;
      T uf_m = u_m * (T(1.0 - 0.5 * xdir) * spd_m) + T(9.81) * h_m * xdir;
      T vf_m = v_m * (T(1.0 - 0.5 * ydir) * spd_m) + T(9.81) * h_m * ydir;
      T a = std::fabs(spd_m + ssign(spd_m) * c_m);
      fh[fid] = T(0.5) * hf_m - T(0.5) * a * (-h_m);
      fu[fid] = T(0.5) * uf_m - T(0.5) * a * (-u_m);
      fv[fid] = T(0.5) * vf_m - T(0.5) * a * (-v_m);
      fz[fid] = h_p / dx;
    } else {
      branch = 4;
      T spd_p = u_p * xdir + v_p * ydir;
      T hf_p = h_p * spd_p;
      T uf_p = u_p * (T(1.0 - 0.5 * xdir) * spd_p) + T(9.81) * h_p * xdir;
      T vf_p = v_p * (T(1.0 - 0.5 * ydir) * spd_p) + T(9.81) * h_p * ydir;
      T a = std::fabs(spd_p + ssign(spd_p) * c_p);
      fh[fid] = T(0.5) * hf_p - T(0.5) * a * (h_p);
      fu[fid] = T(0.5) * uf_p - T(0.5) * a * (u_p);
      fv[fid] = T(0.5) * vf_p - T(0.5) * a * (v_p);
      fz[fid] = h_m / dx;
    }
    fb[fid] = T(branch);
  }

  // SaintVenantTemporalDerivativeKernel::operator() (TemporalDerivativeKernel.cpp:43-99)
  void temporal_derivative(size_t c, const State& S, State& D) {
    auto f = m.adjacent_faces(c);
    double dx = f.dx, dy = f.dy;
    T dhdt = (fh[f.w] - fh[f.e]) / dx + (fh[f.s] - fh[f.n]) / dy;
    T dudt = (fu[f.w] - fu[f.e]) / dx + (fu[f.s] - fu[f.n]) / dy;
    T dvdt = (fv[f.w] - fv[f.e]) / dx + (fv[f.s] - fv[f.n]) / dy;
    dudt += dUdx.h[c] * T(-9.81);
    dvdt += dUdy.h[c] * T(-9.81);
    T dzdx_c = dzdx[c];
    if (std::fabs(dzdx_c) > S.h[c] / dx) dzdx_c = ssign(dzdx_c) * S.h[c] / dx;
    T dzdy_c = dzdy[c];
    if (std::fabs(dzdy_c) > S.h[c] / dy) dzdy_c = ssign(dzdy_c) * S.h[c] / dy;
    T dudt_bed = T(-9.81) * dzdx_c;
    T dvdt_bed = T(-9.81) * dzdy_c;
    dudt += (fz[f.w] - fz[f.e]) / dx;
    dvdt += (fz[f.s] - fz[f.n]) / dy;
    dudt += dudt_bed;
    dvdt += dvdt_bed;
    D.h[c] = dhdt;
    D.u[c] = dudt;
    D.v[c] = dvdt;
  }

  // ManningRoughnessSourceKernel::operator() (ManningRoughnessSourceTerm.cpp:44-88)
  void manning_cell(size_t c, const State& S, State& D, double timestep) {
    T h = S.h[c], u = S.u[c], v = S.v[c];
    T manning_n = smix(ns[c], nd[c], ssmoothstep(ds[c], dd[c], h));
    nh[c] = manning_n;
    if (h > 1e-6) {
      T inv_h = h / (h * h + 1e-3);
      T sf = manning_n * manning_n * std::sqrt(u * u + v * v) * spow43<T>(inv_h);
      Sf[c] = sf;
      T dudt = -T(9.81) * sf * u;
      T dvdt = -T(9.81) * sf * v;
      if (std::fabs(dudt * timestep) > std::fabs(u) && ssign(dudt * timestep) != ssign(u)) dudt = -u / timestep;
      if (std::fabs(dvdt * timestep) > std::fabs(v) && ssign(dvdt * timestep) != ssign(v)) dvdt = -v / timestep;
      D.u[c] += dudt;
      D.v[c] += dvdt;
    } else {
      Sf[c] = 0.0;
    }
  }

  // EnergyLossSourceKernel::operator() (EnergyLossSourceTerm.cpp:56-88)
  void eloss_cell(size_t c, const State& S, State& D, double timestep) {
    T h = S.h[c], u = S.u[c], v = S.v[c];
    if (h > 1e-6) {
      T hyp = std::sqrt(u * u + v * v);
      T dudt = -T(0.5) * u * efx[c] * hyp;
      T dvdt = -T(0.5) * v * efy[c] * hyp;
      if (std::fabs(dudt * timestep) > std::fabs(u) && ssign(dudt * timestep) != ssign(u)) dudt = -u / timestep;
      if (std::fabs(dvdt * timestep) > std::fabs(v) && ssign(dvdt * timestep) != ssign(v)) dvdt = -v / timestep;
      D.u[c] += dudt;
      D.v[c] += dvdt;
    }
  }

  // SmagorinskyCoefficientKernel::operator() (EddyViscositySourceTerm.cpp:97-110) when
  // Smagorinsky, else the coefficient field (or its default); then
  // EddyViscositySourceKernel::operator() (EddyViscositySourceTerm.cpp:46-78). The square
  // pow(x, 2) is taken as x * x. The reference's 0.5 is a double literal, so in FP32 the sum
  // under the root, the root and the products and sum after it are formed in FP64 and the
  // coefficient is rounded once (EddyViscositySourceTerm.cpp:104-108).
  void eddy_cell(size_t c, const State& S, State& D, double timestep) {
    T mu;
    if (p.eddy == 2) {
      T cell_area = T(m.cell_area());
      T a = std::fabs(dUdy.u[c]) + std::fabs(dUdx.v[c]);
      T s = dUdx.u[c] * dUdx.u[c] + dUdy.v[c] * dUdy.v[c];
      mu = T(T(p.eddy_c) + T(p.eddy_s) * cell_area * std::sqrt(s + 0.5 * (a * a)));
    } else {
      mu = emu_set ? emu[c] : T(p.eddy_mu);
    }
    T h = S.h[c], u = S.u[c], v = S.v[c];
    if (h > 1e-6) {
      T dudt = -mu * (d2udx2[c] + d2udy2[c]);
      T dvdt = -mu * (d2vdx2[c] + d2vdy2[c]);
      if (std::fabs(dudt * timestep) > std::fabs(u) && ssign(dudt * timestep) != ssign(u)) dudt = -u / timestep;
      if (std::fabs(dvdt * timestep) > std::fabs(v) && ssign(dvdt * timestep) != ssign(v)) dvdt = -v / timestep;
      D.u[c] += dudt;
      D.v[c] += dvdt;
    }
  }

  // InfiltrationSourceKernel::operator() (InfiltrationSourceTerm.cpp:43-62): the capacity
  // field is consumed at every evaluation, repeated timesteps included.
  void infiltration_cell(size_t c, const State& S, State& D, double timestep) {
    T h = S.h[c];
    T dh = irate[c] * timestep;
    if (dh > h) dh = h;
    if (dh > icap[c]) dh = icap[c];
    D.h[c] -= dh / timestep;
    icap[c] -= dh;
  }

  // DischargeBoundarySourceKernel::operator() (DischargeBoundarySourceTerm.cpp:39-69);
  // returns the depth rate added (0 when skipped).
  T discharge_cell(size_t c, const State& S, State& D, double timestep, double time_now, double step_length) {
    T q0 = qb0[c], q1 = qb1[c];
    if (q0 != 0.0 || q1 != 0.0) {
      T h = S.h[c];
      T dqdt = (q1 - q0) / step_length;
      T qnow = q0 + time_now * dqdt;
      T qnext = qnow + timestep * dqdt;
      T dhdt = T(0.5) * (qnow + qnext);
      if (p.rain_mode == 0) {
        if (h - dhdt * timestep <= 0.0) dhdt = -h / timestep;   // reference clamp (sign quirk)
      } else {
        if (h + dhdt * timestep <= 0.0) dhdt = -h / timestep;   // physical: only stops h < 0
      }
      D.h[c] += dhdt;
      return dhdt;
    }
    return T(0);
  }

  // HeadBoundarySourceKernel::operator() (HeadBoundarySourceTerm.cpp:39-67); returns
  // true when the cell's dh/dt was assigned.
  bool head_cell(size_t c, const State& S, State& D, double timestep, double time_now, double step_length) {
    T h0 = hb0[c], h1 = hb1[c];
    if (forcing.head_kind >= 3) {  // StageBoundarySourceKernel (StageBoundarySourceTerm.cpp:48-52)
      T zc = z[c];
      h0 = hb0[c] - zc;
      h1 = hb1[c] - zc;
    }
    if (!(h0 != h0) && !(h1 != h1)) {
      T h = S.h[c];
      T dhbdydt = (h1 - h0) / step_length;
      T hbdy_now = h0 + time_now * dhbdydt;
      T hbdy_next = hbdy_now + timestep * dhbdydt;
      T target_h = T(0.5) * (hbdy_now + hbdy_next);
      if (target_h <= 0.0) target_h = 0.0;
      T dhdt = (target_h - h) / timestep;
      D.h[c] = dhdt;
      return true;
    }
    return false;
  }

  // SaintVenantSolver::update_dUdt (src/SaintVenant/Solver.cpp:73-114)
  void update_dUdt(size_t state_no, double time_now_d, double timestep_d) override {
    const TT time_now = TT(time_now_d), timestep = TT(timestep_d);
    const State& S = U.at(state_no);
    State& D = K.at(state_no);
    size_t n = m.ncells(), nf = m.nfaces();
    // SaintVenantState::calculate_spatial_derivatives (State.cpp:176-193)
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; ++i) slope_x<T>(m, S.h.data(), dUdx.h.data(), i);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; ++i) slope_x<T>(m, S.u.data(), dUdx.u.data(), i);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; ++i) slope_x<T>(m, S.v.data(), dUdx.v.data(), i);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; ++i) slope_y<T>(m, S.h.data(), dUdy.h.data(), i);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; ++i) slope_y<T>(m, S.u.data(), dUdy.u.data(), i);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; ++i) slope_y<T>(m, S.v.data(), dUdy.v.data(), i);
    // SaintVenantFluxes::update (Fluxes.cpp:44-65)
#pragma omp parallel for schedule(static)
    for (size_t f = 0; f < nf; ++f) flux_face(f, S);
    // temporal derivative (Solver.cpp:88-95)
#pragma omp parallel for schedule(static)
    for (size_t c = 0; c < n; ++c) temporal_derivative(c, S, D);
    // source terms (Solver.cpp:98-104)
    // (energy loss and infiltration run when both of their fields were set, as the
    // reference constructs each with both fields; Manning and energy loss in their
    // configuration order, infiltration touches dh/dt only)
    auto run_manning = [&]() {
      if (!p.manning) return;
#pragma omp parallel for schedule(static)
      for (size_t c = 0; c < n; ++c) manning_cell(c, S, D, double(timestep));
    };
    auto run_eloss = [&]() {
      if ((present & 12u) != 12u) return;
#pragma omp parallel for schedule(static)
      for (size_t c = 0; c < n; ++c) eloss_cell(c, S, D, double(timestep));
    };
    auto run_eddy = [&]() {
      if (!p.eddy) return;
      // second derivatives: Minmod3 of the slopes along the same axis
      // (EddyViscositySourceTerm.hpp:222-228)
#pragma omp parallel for schedule(static)
      for (size_t i = 0; i < n; ++i) slope_x<T>(m, dUdx.u.data(), d2udx2.data(), i);
#pragma omp parallel for schedule(static)
      for (size_t i = 0; i < n; ++i) slope_y<T>(m, dUdy.u.data(), d2udy2.data(), i);
#pragma omp parallel for schedule(static)
      for (size_t i = 0; i < n; ++i) slope_x<T>(m, dUdx.v.data(), d2vdx2.data(), i);
#pragma omp parallel for schedule(static)
      for (size_t i = 0; i < n; ++i) slope_y<T>(m, dUdy.v.data(), d2vdy2.data(), i);
#pragma omp parallel for schedule(static)
      for (size_t c = 0; c < n; ++c) eddy_cell(c, S, D, double(timestep));
    };
    int order[3] = {p.term_order[0], p.term_order[1], p.term_order[2]};
    if (!p.order_set && p.eloss_first) { order[0] = 2; order[1] = 1; }
    for (int t : order) {
      if (t == 1) run_manning();
      else if (t == 2) run_eloss();
      else run_eddy();
    }
    if ((present & 3u) == 3u) {
#pragma omp parallel for schedule(static)
      for (size_t c = 0; c < n; ++c) infiltration_cell(c, S, D, double(timestep));
    }
    // boundaries in configuration order (Solver.cpp:107-113); the tallies record the rain
    // depth rate added and the depth rate removed by the head assignment.
    const double L = double(p.step_duration);
    if (!track_tallies) {
      auto run_discharge = [&]() {
#pragma omp parallel for schedule(static)
        for (size_t c = 0; c < n; ++c) discharge_cell(c, S, D, double(timestep), double(time_now), L);
      };
      auto run_head = [&]() {
#pragma omp parallel for schedule(static)
        for (size_t c = 0; c < n; ++c) head_cell(c, S, D, double(timestep), double(time_now), L);
      };
      if (p.head_first) { run_head(); run_discharge(); }
      else { run_discharge(); run_head(); }
      return;
    }
    std::vector<double> rain(n, 0.0), removed(n, 0.0), wall(n, 0.0);
    // flow through the mesh-edge faces (before any boundary assignment)
#pragma omp parallel for schedule(static)
    for (size_t c = 0; c < n; ++c) {
      auto f = m.adjacent_faces(c);
      size_t x = c % m.nx, y = c / m.nx;
      double w = 0.0;
      if (x == 0) w += double(T(fh[f.w] / f.dx));
      if (x == m.nx - 1) w -= double(T(fh[f.e] / f.dx));
      if (y == 0) w += double(T(fh[f.s] / f.dy));
      if (y == m.ny - 1) w -= double(T(fh[f.n] / f.dy));
      wall[c] = w;
    }
    auto run_discharge = [&]() {
#pragma omp parallel for schedule(static)
      for (size_t c = 0; c < n; ++c) rain[c] = double(discharge_cell(c, S, D, double(timestep), double(time_now), L));
    };
    auto run_head = [&]() {
#pragma omp parallel for schedule(static)
      for (size_t c = 0; c < n; ++c) {
        T before = D.h[c];
        if (head_cell(c, S, D, double(timestep), double(time_now), L)) removed[c] = double(before) - double(D.h[c]);
      }
    };
    if (p.head_first) { run_head(); run_discharge(); }
    else { run_discharge(); run_head(); }
    rain_sum_[state_no] = neumaier_sum(rain.data(), n);
    out_sum_[state_no] = neumaier_sum(removed.data(), n);
    wall_sum_[state_no] = neumaier_sum(wall.data(), n);
  }

  // RungeKuttaSolver::update_y (src/TemporalScheme/RungeKutta.hpp:371-405)
  void update_y(size_t step, TT timestep) {
    size_t n = m.ncells();
    State& Y = U.at(step);
    const State& U0 = U.at(0);
    Y.h = U0.h; Y.u = U0.u; Y.v = U0.v;
    for (size_t col = 0; col < step; ++col) {
      const T coef = T(tab.A(step + 1, col + 1) * timestep);
      const State& Kc = K.at(col);
#pragma omp parallel for schedule(static)
      for (size_t i = 0; i < n; ++i) {
        Y.h[i] += Kc.h[i] * coef;
        Y.u[i] += Kc.u[i] * coef;
        Y.v[i] += Kc.v[i] * coef;
      }
    }
  }

  // SaintVenantState::max_control_number (src/SaintVenant/State.cpp:195-230)
  T control_number(size_t state_no, double timestep) const {
    const State& S = U.at(state_no);
    size_t n = m.ncells();
    const T dx = m.dx, dy = m.dy;
    T max_cn = 0.0;
    bool any_nan = false;
#pragma omp parallel
    {
      T local = 0.0;
      bool lnan = false;
#pragma omp for schedule(static)
      for (size_t i = 0; i < n; ++i) {
        T h = sfmax(S.h[i], T(0.0));
        T u = std::fabs(S.u[i]);
        T v = std::fabs(S.v[i]);
        T c = std::sqrt(T(9.81) * h);
        T cn = timestep * (((u + c) / dx) + ((v + c) / dy));
        if (cn != cn) lnan = true;
        else if (cn > local) local = cn;
      }
#pragma omp critical
      {
        if (local > max_cn) max_cn = local;
        any_nan = any_nan || lnan;
      }
    }
    return any_nan ? std::numeric_limits<T>::quiet_NaN() : max_cn;
  }

  // RungeKuttaTemporalScheme::do_timestep (src/TemporalScheme/RungeKutta.cpp:141-167),
  // with the target control number as a parameter (the reference hard-codes 1.0; for 1.0
  // the generalised expressions below are bit-identical to the reference's).
  void do_timestep(double local_time_d, double dt_d, double* cn_out, int* repeat, double* new_dt) override {
    const TT local_time = TT(local_time_d), dt = TT(dt_d);
    size_t N = tab.nsteps();
    for (size_t substep = 1; substep <= N; ++substep) {
      TT substep_time = local_time + tab.c(substep) * dt;
      update_dUdt(substep - 1, double(substep_time), double(dt));  // update_k
      update_y(substep, dt);
    }
    const double cn_target = p.cn_target;
    double cn = double(control_number(N, double(dt)));
    *cn_out = cn;
    TT nd;
    int rep;
    if (cn > cn_target) {
      rep = 1;
      nd = (cn > 5.0 * cn_target) ? TT(dt / 5.0) : TT((dt * cn_target) / (cn * 1.1));
    } else if (cn > 0.9 * cn_target) {
      rep = 0; nd = TT(dt);
    } else {
      rep = 0; nd = TT((dt * cn_target) / cn);
    }
    if (p.max_dt > 0.0 && nd > TT(p.max_dt)) nd = TT(p.max_dt);
    *repeat = rep;
    *new_dt = double(nd);
  }

  // RungeKuttaSolver::accept_timestep (RungeKutta.hpp:428-431)
  void accept() override {
    size_t N = tab.nsteps();
    U[0].h = U[N].h; U[0].u = U[N].u; U[0].v = U[N].v;
  }

  // Weighted tally of the last timestep's stages: sum_s b_s dt * (sum over cells) * area.
  void add_tallies(TT dt) {
    size_t N = tab.nsteps();
    double area = m.cell_area();
    for (size_t s = 0; s < N; ++s) {
      double w = double(T(tab.b(s + 1) * dt));
      st_.rain_in += w * rain_sum_[s] * area;
      st_.outflow += w * out_sum_[s] * area;
      st_.wall_in += w * wall_sum_[s] * area;
    }
  }

  // TypedTemporalScheme::step (src/TemporalScheme/TemporalScheme.hpp:112-149)
  void step(Stats* out) override {
    TT t_local = 0.0;
    TT step_duration = TT(p.step_duration);
    uint64_t acc0 = st_.accepted, rep0 = st_.repeated;
    while (t_local < step_duration) {
      double cn, nd_d;
      int repeat;
      do_timestep(double(t_local), double(dt_), &cn, &repeat, &nd_d);
      TT new_dt = TT(nd_d);
      if (repeat) {
        st_.repeated++;
      } else {
        st_.accepted++;
        if (track_tallies) add_tallies(dt_);
        t_local += dt_;
        accept();
      }
      dt_ = new_dt;
      if (t_local >= step_duration) break;
      else if (t_local + dt_ > step_duration) dt_ = step_duration - t_local;
      else if (t_local + 2.0 * dt_ > step_duration) dt_ = (step_duration - t_local) * 0.4;
    }
    if (out) {
      *out = st_;
      out->accepted = st_.accepted - acc0;
      out->repeated = st_.repeated - rep0;
      out->volume = volume();
    }
  }

  // SaintVenantVolumeMeasure::get_volume (src/SaintVenant/Measure.hpp:137-156), summed in
  // FP64 in a fixed order with compensation.
  double volume() const override {
    size_t n = m.ncells();
    std::vector<double> hv(n);
    double area = m.cell_area();
    for (size_t i = 0; i < n; ++i) hv[i] = double(U[0].h[i]) * area;
    return neumaier_sum(hv.data(), n);
  }
};

}  // namespace svo
