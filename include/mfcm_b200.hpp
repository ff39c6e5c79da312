// mfcm_b200.hpp -- C++ facade over the C-ABI in sv.h, named after the reference's classes.
//
// The reference drives its time step through RungeKuttaSolver<SaintVenantSolver<TT, T,
// Cartesian2DMesh>> (src/mfcm.cpp:19-36). These header-only classes keep those names, the
// template parameters that matter (TT time type, T value type), the member functions the
// reference's loop calls (update_dUdt, state, dUdt, start_new_step, end_of_step,
// do_timestep, accept_timestep, step, solve) and its error convention (std::runtime_error),
// so host code written against the reference's solver can be pointed at the B200 library.
// Every call goes through libsv_b200.so; nothing here computes the scheme on the host.
//
// Differences a porter should know:
//  * Fields live on the device. State and derivative accessors return host copies
//    (std::vector<double>) and field setters upload; the reference's sycl::buffer-backed
//    Field/DataArray objects have no device-side equivalent here.
//  * Boundary values are passed per step through start_new_step (rain as a TimeSeries or a
//    per-cell pattern, outflow as a head target on mesh edges) instead of being read from
//    the .mf configuration.
//  * T = double is the FP64 path (bit-for-bit the reference arithmetic at T = double);
//    T = float is FP32 state with FP64 reductions, optionally with the bed stored as FP32
//    offsets from FP64 tile datums (Options::datum64).
#ifndef MFCM_B200_HPP
#define MFCM_B200_HPP

#include <cstddef>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "sv.h"

namespace mfcm_b200 {

// Throws std::runtime_error with the library's message for a non-zero status, the way the
// reference reports failures (e.g. src/SpatialDerivative/SpatialDerivative.cpp:49-56).
inline void check(int rc, const sv_ctx* ctx = nullptr) {
  if (rc != SV_OK) throw std::runtime_error(std::string("mfcm_b200: ") + sv_last_error(ctx));
}

// Cartesian2DMesh (src/Mesh/Cartesian2DMesh.hpp): cell counts, spacing and origin; cells
// are numbered i = y * nx + x (Cartesian2DMesh.hpp:143-145); vertical faces come first,
// then horizontal faces (Cartesian2DMesh.hpp:379-435).
class Cartesian2DMesh {
 public:
  Cartesian2DMesh(uint64_t nx, uint64_t ny, double dx, double dy, double origin_x = 0.0, double origin_y = 0.0)
      : d_{nx, ny, dx, dy, origin_x, origin_y} {
    if (nx == 0 || ny == 0 || !(dx > 0.0) || !(dy > 0.0))
      throw std::runtime_error("Cartesian2DMesh: cell count and cell size must be positive");
  }
  uint64_t nxcells() const { return d_.nx; }
  uint64_t nycells() const { return d_.ny; }
  double dx() const { return d_.dx; }
  double dy() const { return d_.dy; }
  uint64_t cell_count() const { return d_.nx * d_.ny; }
  uint64_t face_count() const { return (d_.nx + 1) * d_.ny + (d_.ny + 1) * d_.nx; }
  uint64_t cell_id(uint64_t x, uint64_t y) const { return y * d_.nx + x; }
  const sv_mesh_desc& desc() const { return d_; }

 private:
  sv_mesh_desc d_;
};

// TimeParameters / RungeKuttaTimeParameters (src/Config/TimeParameters.cpp:21-58).
struct TimeParameters {
  double start_time = 0.0;
  double end_time = 0.0;
  double step_duration = 60.0;     // "step duration seconds"
  double initial_timestep = 1.0;   // "initial timestep seconds"
  // TimeParameters::num_steps (TimeParameters.cpp:40-58): whole steps, with the end time
  // accepted when it lies within 1e-6 s of a step boundary
  std::size_t num_steps() const {
    const double eps = 1e-6;
    double sim = end_time - start_time;
    std::size_t n = static_cast<std::size_t>(sim / step_duration);
    if (step_duration * double(n) >= sim - eps && step_duration * double(n) <= sim + eps) return n;
    return n + 1;
  }
};

// TimeSeries<double,double>::at with linear interpolation (src/Input/TimeSeries.cpp:26-47);
// beyond the last knot the last segment is extrapolated.
class TimeSeries {
 public:
  TimeSeries(std::vector<double> t, std::vector<double> v) : t_(std::move(t)), v_(std::move(v)) {
    if (t_.size() < 2 || t_.size() != v_.size())
      throw std::runtime_error("TimeSeries: at least two (time, value) knots are needed");
  }
  static TimeSeries constant(double v) { return TimeSeries({0.0, 1.0}, {v, v}); }
  double at(double time) const {
    std::size_t i1 = 1;
    while (i1 < t_.size() && !(t_[i1] > time)) ++i1;
    if (i1 >= t_.size()) i1 = t_.size() - 1;
    const std::size_t i0 = i1 - 1;
    const double dvdt = (v_[i1] - v_[i0]) / (t_[i1] - t_[i0]);
    return v_[i0] + dvdt * (time - t_[i0]);
  }

 private:
  std::vector<double> t_, v_;
};

// Field ids of sv.h (SaintVenantState / SaintVenantConstants / source-term fields).
enum class FieldId : int {
  z_bed = SV_FIELD_Z, h = SV_FIELD_H, u = SV_FIELD_U, v = SV_FIELD_V,
  n_shallow = SV_FIELD_N_SHALLOW, n_deep = SV_FIELD_N_DEEP, d_shallow = SV_FIELD_D_SHALLOW,
  d_deep = SV_FIELD_D_DEEP, qbdy0 = SV_FIELD_QBDY0, qbdy1 = SV_FIELD_QBDY1, hbdy0 = SV_FIELD_HBDY0,
  hbdy1 = SV_FIELD_HBDY1, rain_pattern = SV_FIELD_RAIN_PATTERN, dzdx_bed = SV_FIELD_DZDX,
  dzdy_bed = SV_FIELD_DZDY, hflux = SV_FIELD_FLUX_H, uflux = SV_FIELD_FLUX_U, vflux = SV_FIELD_FLUX_V,
  zflux = SV_FIELD_FLUX_Z, branch = SV_FIELD_FLUX_BRANCH, infil_rate = SV_FIELD_INFIL_RATE,
  infil_cap = SV_FIELD_INFIL_CAP, eloss_fx = SV_FIELD_ELOSS_FX, eloss_fy = SV_FIELD_ELOSS_FY,
  eddy_mu = SV_FIELD_EDDY_MU
};

// Host copy of one SaintVenantState (src/SaintVenant/State.hpp:40-42).
struct StateCopy {
  std::vector<double> h, u, v;
};

// Solver options that the reference reads from its configuration file.
struct Options {
  double cn_target = 1.0;        // the reference hard-codes 1.0 (RungeKutta.cpp:154)
  double max_dt = 0.0;           // 0: no clamp (reference behaviour)
  bool physical_rain_clamp = false;  // false: the reference's discharge clamp
  bool manning = true;           // "manning roughness" source term present
  bool head_first = false;       // head boundary listed before the discharge boundary
  bool datum64 = false;          // T = float only: bed as FP32 offsets from FP64 tile datums
  bool tallies = true;           // FP64 rain / outflow volume tallies
  int device = 0;
};

// Boundary values for one step (start_new_step of the discharge and head boundaries,
// DischargeBoundarySourceTerm.hpp:114-146, HeadBoundarySourceTerm.hpp:114-146).
struct StepBoundaries {
  enum class Rain { none, uniform, pattern } rain_kind = Rain::none;
  const TimeSeries* rain = nullptr;   // m/s (uniform, or multiplying the per-cell pattern)
  bool head = false;                  // head target on whole mesh edges
  unsigned head_edges = 0;            // SV_EDGE_* bits
  const TimeSeries* head_level = nullptr;
};

// SaintVenantSolver<TT, T, Mesh> (src/SaintVenant/Solver.hpp:30-172) over one sv_ctx.
template <typename TT, typename T, typename Mesh = Cartesian2DMesh>
class SaintVenantSolver {
  static_assert(std::is_same<T, double>::value || std::is_same<T, float>::value,
                "SaintVenantSolver: T must be double or float");

 public:
  using TimeType = TT;
  using ValueType = T;
  using MeshType = Mesh;

  SaintVenantSolver(std::shared_ptr<MeshType> mesh, std::shared_ptr<TimeParameters> tparams, int rk_method,
                    const Options& opt = Options())
      : mesh_(std::move(mesh)), tparams_(std::move(tparams)) {
    sv_params p{};
    p.precision = std::is_same<T, double>::value ? SV_F64 : (opt.datum64 ? SV_F32_DATUM64 : SV_F32);
    p.rk_method = rk_method;
    p.cn_target = opt.cn_target;
    p.step_duration = tparams_->step_duration;
    p.initial_dt = tparams_->initial_timestep;
    p.max_dt = opt.max_dt;
    p.rain_mode = opt.physical_rain_clamp ? 1 : 0;
    p.manning = opt.manning ? 1 : 0;
    p.head_first = opt.head_first ? 1 : 0;
    p.flags = opt.tallies ? 0 : SV_FLAG_NO_TALLIES;
    sv_ctx* c = nullptr;
    check(sv_create(&mesh_->desc(), &p, opt.device, &c), nullptr);
    ctx_.reset(c);
  }

  const MeshType& mesh() const { return *mesh_; }
  sv_ctx* handle() { return ctx_.get(); }

  // field upload / download (SaintVenantConstants, U_[0], source-term fields)
  void set_field(FieldId id, const std::vector<double>& host) {
    check(sv_set_field(ctx_.get(), int(id), host.data(), host.size()), ctx_.get());
  }
  std::vector<double> get_field(FieldId id) const {
    bool face = int(id) >= SV_FIELD_FLUX_H && int(id) <= SV_FIELD_FLUX_BRANCH;
    std::vector<double> out(face ? mesh_->face_count() : mesh_->cell_count());
    check(sv_get_field(ctx_.get(), int(id), out.data(), out.size()), ctx_.get());
    return out;
  }
  // ManningRoughnessSourceTerm uniform parameters (ManningRoughnessSourceTerm.cpp:90-109)
  void set_manning(double n_shallow, double n_deep, double d_shallow, double d_deep) {
    check(sv_set_manning(ctx_.get(), n_shallow, n_deep, d_shallow, d_deep), ctx_.get());
  }

  // EddyViscositySourceTerm (EddyViscositySourceTerm.cpp:112-137): SV_EDDY_CONSTANT with
  // "default mu" (or the eddy_mu field), SV_EDDY_SMAGORINSKY with the constant and dynamic
  // coefficients
  void set_eddy_viscosity(int mode, double mu = 1.0, double mu_const = 0.05, double mu_smag = 0.5) {
    check(sv_set_eddy_viscosity(ctx_.get(), mode, mu, mu_const, mu_smag), ctx_.get());
  }
  // the momentum source terms (SV_TERM_*) in the order of the configuration's source terms
  void set_source_order(const std::vector<int>& terms) {
    check(sv_set_source_order(ctx_.get(), terms.data(), int(terms.size())), ctx_.get());
  }

  // SaintVenantSolver::update_dUdt (Solver.cpp:73-114)
  void update_dUdt(std::size_t state_no, const TT& time_now, const TT& timestep) {
    check(sv_eval_dudt(ctx_.get(), int(state_no), double(time_now), double(timestep)), ctx_.get());
  }
  // SaintVenantSolver::start_new_step (Solver.cpp:116-129) with this step's boundary values
  void start_new_step(const TT& time_now, const StepBoundaries& b) {
    const double t0 = double(time_now), t1 = double(time_now) + tparams_->step_duration;
    sv_forcing f{};
    if (b.rain_kind != StepBoundaries::Rain::none && b.rain) {
      f.rain_kind = b.rain_kind == StepBoundaries::Rain::uniform ? SV_RAIN_UNIFORM : SV_RAIN_PATTERN;
      f.rain_q0 = b.rain->at(t0);
      f.rain_q1 = b.rain->at(t1);
    }
    if (b.head) {
      f.head_kind = SV_HEAD_EDGES;
      f.head_edges = b.head_edges;
      f.head_h0 = b.head_level ? b.head_level->at(t0) : 0.0;
      f.head_h1 = b.head_level ? b.head_level->at(t1) : 0.0;
    }
    check(sv_set_forcing(ctx_.get(), &f), ctx_.get());
  }
  // SaintVenantSolver::end_of_step (Solver.hpp:90-98): the measures are the FP64 tallies
  sv_stats end_of_step(const TT&) {
    sv_stats s{};
    check(sv_get_stats(ctx_.get(), &s), ctx_.get());
    return s;
  }
  // SaintVenantSolver::state(i) / dUdt(i) (Solver.hpp:100-115), as host copies
  StateCopy state(std::size_t i = 0) const { return copy(SV_FIELD_STATE_BASE + 3 * int(i)); }
  StateCopy dUdt(std::size_t i) const { return copy(SV_FIELD_K_BASE + 3 * int(i)); }
  void set_state(const StateCopy& s) {
    set_field(FieldId::h, s.h);
    set_field(FieldId::u, s.u);
    set_field(FieldId::v, s.v);
  }

 private:
  struct Deleter {
    void operator()(sv_ctx* c) const { sv_destroy(c); }
  };
  StateCopy copy(int base) const {
    StateCopy s;
    std::vector<double>* f[3] = {&s.h, &s.u, &s.v};
    for (int k = 0; k < 3; ++k) {
      f[k]->resize(mesh_->cell_count());
      check(sv_get_field(ctx_.get(), base + k, f[k]->data(), f[k]->size()), ctx_.get());
    }
    return s;
  }
  std::shared_ptr<MeshType> mesh_;
  std::shared_ptr<TimeParameters> tparams_;
  std::unique_ptr<sv_ctx, Deleter> ctx_;
};

// runge_kutta_named_coefficient_sets_ (src/TemporalScheme/RungeKutta.cpp:54-115) by name
inline int named_coefficient_set(const std::string& name) {
  static const char* names[] = {"euler", "midpoint", "heun2", "ralston2", "kutta3", "heun3",
                                "wray3", "ralston3", "ssprk3", "classic", "ralston4", "3/8rule"};
  for (int i = 0; i < 12; ++i)
    if (name == names[i]) return i;
  throw std::runtime_error("unknown Runge-Kutta coefficient set: " + name);
}

// RungeKuttaSolver<Solver> (src/TemporalScheme/RungeKutta.hpp:268-463) with the step loop of
// TypedTemporalScheme (src/TemporalScheme/TemporalScheme.hpp:112-149,244-276).
template <typename Solver>
class RungeKuttaSolver {
 public:
  using TimeType = typename Solver::TimeType;
  using SolverType = Solver;
  struct timestep_result {
    TimeType new_dt;
    bool repeat_timestep;
    double control_number;
  };
  struct step_result {
    std::size_t num_timesteps;
    std::size_t num_repeated_timesteps;
  };

  RungeKuttaSolver(std::shared_ptr<TimeParameters> tparams, const std::string& named_coeffs,
                   std::shared_ptr<typename Solver::MeshType> mesh, const Options& opt = Options())
      : tparams_(tparams),
        solver_(std::make_shared<Solver>(std::move(mesh), tparams, named_coefficient_set(named_coeffs), opt)) {}

  SolverType& solver() { return *solver_; }

  // RungeKuttaTemporalScheme::do_timestep (RungeKutta.cpp:141-167): stages into U_[N], the
  // control number and the next dt; U_[0] is unchanged until accept_timestep
  timestep_result do_timestep(const TimeType& local_time, const TimeType& dt) {
    double cn = 0.0, nd = 0.0;
    int rep = 0;
    check(sv_do_timestep(solver_->handle(), double(local_time), double(dt), &cn, &rep, &nd), solver_->handle());
    return {TimeType(nd), rep != 0, cn};
  }
  // RungeKuttaSolver::accept_timestep (RungeKutta.hpp:424-431)
  void accept_timestep() { check(sv_accept(solver_->handle()), solver_->handle()); }
  // TypedTemporalScheme::step (TemporalScheme.hpp:112-149): the adaptive-dt loop of one step,
  // run on the device
  step_result step() {
    sv_stats s{};
    check(sv_advance(solver_->handle(), &s), solver_->handle());
    return {std::size_t(s.accepted), std::size_t(s.repeated)};
  }
  // the dt carried into the next timestep (dt_ of the reference's scheme)
  TimeType current_timestep() {
    double dt = 0.0;
    check(sv_get_dt(solver_->handle(), &dt), solver_->handle());
    return TimeType(dt);
  }
  // TypedTemporalScheme::solve (TemporalScheme.hpp:244-276): start_new_step, step and
  // end_of_step for every step from start_time to end_time; `boundaries(t)` supplies each
  // step's boundary values
  template <typename BoundaryFn>
  std::vector<step_result> solve(BoundaryFn&& boundaries) {
    std::vector<step_result> out;
    const std::size_t n = tparams_->num_steps();
    for (std::size_t i = 0; i < n; ++i) {
      TimeType t = TimeType(tparams_->start_time + double(i) * tparams_->step_duration);
      solver_->start_new_step(t, boundaries(t));
      out.push_back(step());
      solver_->end_of_step(t + TimeType(tparams_->step_duration));
    }
    return out;
  }

 private:
  std::shared_ptr<TimeParameters> tparams_;
  std::shared_ptr<Solver> solver_;
};

}  // namespace mfcm_b200

#endif  // MFCM_B200_HPP
