// ref_pin.cpp -- TEST INFRASTRUCTURE: runs the reference's own hot-path code on the CPU so that
// the oracle (oracle/sv_oracle.hpp) can be checked against it. Built by oracle/ref_pin/build.py
// into oracle/_ref/libsv_refpin.so from the reference's sources; only tests/ load it.
//
// What runs here is the reference's code, compiled unchanged:
//   mesh, field and data-array classes    src/Mesh/Cartesian2DMesh.hpp and .cpp (the configured
//                                         constructor, cell centres and cell lookups),
//                                         src/Field/Field.cpp, src/DataArray/DataArray.cpp
//   slopes                                SaintVenantState::calculate_spatial_derivatives
//                                         (src/SaintVenant/State.cpp:176-193) with
//                                         SpatialDerivativeOperator<Minmod3> (SpatialDerivative.cpp)
//   bed slopes                            the same operator on z (as Constants.cpp:39-40)
//   face fluxes                           SaintVenantFluxes::update (Fluxes.cpp) launching
//                                         SaintVenantFluxKernel (FluxKernel.cpp:62-295)
//   temporal derivative                   SaintVenantTemporalDerivativeKernel (:43-99)
//   Manning roughness                     ManningRoughnessSourceKernel (:44-88)
//   discharge and head boundaries         DischargeBoundarySourceKernel (:39-69),
//                                         HeadBoundarySourceKernel (:39-67)
//   further source and boundary terms     EnergyLossSourceKernel (EnergyLossSourceTerm.cpp),
//                                         InfiltrationSourceKernel (InfiltrationSourceTerm.cpp),
//                                         EddyViscositySourceKernel and SmagorinskyCoefficientKernel
//                                         with the second derivatives of EddyViscositySourceTerm::
//                                         apply (EddyViscositySourceTerm.hpp:222-257),
//                                         StageBoundarySourceKernel (StageBoundarySourceTerm.cpp)
//   output file formats                   CSVOutput and RawBinaryOutput (src/Output/OutputFormat.hpp)
//                                         over FieldOutputFunction (cell fields with their
//                                         locations) and TimeSeriesOutputFunction (measures),
//                                         src/Output/OutputFunction.hpp
//   control number                        SaintVenantState::max_control_number (State.cpp:195-230)
//   stage combination                     the SaintVenantState operators (State.cpp:88-174) in
//                                         the order of RungeKuttaSolver::update_y
//                                         (RungeKutta.hpp:377-388)
//   whole solves                          RungeKuttaSolver<Solver> (RungeKutta.hpp:268-463) with
//                                         the named tableaux and do_timestep (RungeKutta.cpp),
//                                         TypedTemporalScheme::solve / step (TemporalScheme.hpp)
//                                         and TimeParameters::num_steps (TimeParameters.cpp)
// The driver only creates the objects, fills them from arrays and launches the kernels in the
// order of SaintVenantSolver::update_dUdt (Solver.cpp:73-114) -- the launch code of each
// source and boundary term's apply() -- and copies the results out. For whole solves it
// stands in for SaintVenantSolver (whose constructor reads the configuration) with PinSolver,
// which has the same interface and sets the boundary values as the discharge and head terms'
// start_new_step do for a global rain selection and edge-strip head selections.
#include "sycl.hpp"

#include "DataArray.hpp"
#include "DataArray.cpp"
#include "Mesh.hpp"
#include "Cartesian2DMesh.hpp"
#include "MeshSelection.hpp"
#include "Field.hpp"
#include "Field.cpp"
#include "FieldOperators.cpp"
#include "Minmod3.hpp"
#include "SpatialDerivative.hpp"
#include "SpatialDerivative.cpp"
#include "State.hpp"
#include "Constants.hpp"
#include "State.cpp"
#include "Fluxes.hpp"
#include "Fluxes.cpp"
#include "FluxKernel.cpp"
#include "TemporalDerivativeKernel.hpp"
#include "TemporalDerivativeKernel.cpp"
#include "SourceTerm.hpp"
#include "ManningRoughnessSourceTerm.hpp"
#include "ManningRoughnessSourceTerm.cpp"
#include "DischargeBoundarySourceTerm.hpp"
#include "DischargeBoundarySourceTerm.cpp"
#include "HeadBoundarySourceTerm.hpp"
#include "HeadBoundarySourceTerm.cpp"
#include "EnergyLossSourceTerm.hpp"
#include "EnergyLossSourceTerm.cpp"
#include "InfiltrationSourceTerm.hpp"
#include "InfiltrationSourceTerm.cpp"
#include "EddyViscositySourceTerm.hpp"
#include "EddyViscositySourceTerm.cpp"
#include "StageBoundarySourceTerm.hpp"
#include "StageBoundarySourceTerm.cpp"
#include "TimeParameters.hpp"
#include "TimeParameters.cpp"
#include "RungeKutta.hpp"
#include "RungeKutta.cpp"
#include "OutputFunction.hpp"
#include "OutputFormat.hpp"

#include <cstdint>
#include <cstring>
#include <iostream>

// ---- glue the reference defines in files that read its configuration --------------------
// Cartesian2DMesh's configured constructor, device moves and accessor are the reference's own
// (src/Mesh/Cartesian2DMesh.cpp, compiled below with the configuration stand-in).
#include "Cartesian2DMesh.cpp"

// MeshSelection, global selections only (MeshSelection.cpp:22-33, 146-157, 196-214): a global
// selection is a two-entry list holding the object count twice.
template <typename Mesh, MeshComponent C>
MeshSelection<Mesh, C>::MeshSelection(const std::shared_ptr<MeshType>& mesh_p, const Config&)
    : mesh_p_(mesh_p), list_(mesh_p->queue_ptr(), 0) {
  initialize_global_();
}
template <typename Mesh, MeshComponent C>
void MeshSelection<Mesh, C>::initialize_global_(void) {
  std::vector<size_t>& id_list = list_.host_vector();
  size_t idmax = mesh_p_->template object_count<FieldMappingType>();
  id_list.push_back(idmax);
  id_list.push_back(idmax);
  list_.move_to_device();
}
template <typename Mesh, MeshComponent C>
bool MeshSelection<Mesh, C>::is_global(void) const {
  return list_.size() == 2 && list_.host_vector().at(0) == list_.host_vector().at(1);
}
template <typename Mesh, MeshComponent C>
size_t MeshSelection<Mesh, C>::size(void) const {
  if (is_global()) return mesh_p_->template object_count<FieldMappingType>();
  return list_.size() - 1;
}

// SaintVenantConstants (Constants.cpp:25-44) with the bed taken from an array instead of a
// configured field generator; the slopes come from the reference's operator as there.
template <typename T>
struct PinBed {
  static std::vector<T> z;
};
template <typename T>
std::vector<T> PinBed<T>::z;
template <typename T, typename Mesh>
SaintVenantConstants<T, Mesh>::SaintVenantConstants(const std::shared_ptr<MeshType>& mesh, bool on_device)
    : mesh_(mesh),
      z_bed_(mesh_->queue_ptr(), "z_bed", mesh_, PinBed<T>::z, on_device),
      dzdx_bed_(mesh_->queue_ptr(), "dzdx_bed", mesh_, 0.0f, on_device),
      dzdy_bed_(mesh_->queue_ptr(), "dzdy_bed", mesh_, 0.0f, on_device) {
  using SpatialDerivative = SpatialDerivativeOperator<ValueType, MeshType, MeshComponent::Cell, Minmod3<ValueType>>;
  SpatialDerivative::template apply<SpatialDerivativeAxis::X>(z_bed_, dzdx_bed_);
  SpatialDerivative::template apply<SpatialDerivativeAxis::Y>(z_bed_, dzdy_bed_);
}

std::shared_ptr<sycl::queue> get_sycl_queue(void) { return std::make_shared<sycl::queue>(); }

namespace {

template <typename T>
using CF = CellField<T, Cartesian2DMesh>;
template <typename T>
using State = SaintVenantState<T, Cartesian2DMesh>;

std::shared_ptr<Cartesian2DMesh> make_mesh(const std::shared_ptr<sycl::queue>& q, uint64_t nx, uint64_t ny, double dx,
                                           double dy) {
  Config& c = GlobalConfig::instance().mesh;
  c.kv.clear();
  c.kv["cell count"] = std::to_string(nx) + ", " + std::to_string(ny);
  {
    std::ostringstream s;
    s.precision(17);
    s << dx << ", " << dy;
    c.kv["cell size"] = s.str();
  }
  return std::make_shared<Cartesian2DMesh>(q, true);
}

template <typename T>
std::vector<T> vec(const T* p, size_t n) {
  return std::vector<T>(p, p + n);
}

// a field's values: move it to the host (DataArray::move_to_host writes the buffer back), copy
template <typename F, typename T>
void read(F& f, T* out) {
  f.move_to_host();
  const std::vector<T>& v = f.data().host_vector();
  std::copy(v.begin(), v.end(), out);
  f.move_to_device();
}

template <typename T>
void set_state(State<T>& s, const std::shared_ptr<sycl::queue>& q, const std::shared_ptr<Cartesian2DMesh>& m,
               const T* h, const T* u, const T* v, size_t n) {
  s.h() = CF<T>(q, "h", m, vec(h, n), true);
  s.u() = CF<T>(q, "u", m, vec(u, n), true);
  s.v() = CF<T>(q, "v", m, vec(v, n), true);
}

// One update_dUdt (Solver.cpp:73-114) of the state (h, u, v) on bed z, at local time
// `time_now` with `timestep` and step length `step_length` (rounded to T first, as TimeType). Optional terms are
// skipped when their arrays are null: Manning (ns, nd, ds, dd), discharge (q0, q1), head
// (hb0, hb1), in the configured order (head before discharge when head_first).
// out: dzdx, dzdy, dhdx, dudx, dvdx, dhdy, dudy, dvdy (cell fields), then h, u, v, z flux and
// branch (face fields), then dh/dt, du/dt, dv/dt (cell fields).
template <typename T>
int dudt(uint64_t nx, uint64_t ny, double dx, double dy, const T* z, const T* h, const T* u, const T* v, const T* ns,
         const T* nd, const T* ds, const T* dd, const T* q0, const T* q1, const T* hb0, const T* hb1, int head_first,
         double time_now, double timestep, double step_length, T* out) {
  try {
    // the shipped solver takes its times in the value type (TimeType = ValueType, mfcm.cpp:13-16):
    // the kernels receive them widened from T
    using TT = T;
    const TT tnow = TT(time_now), tstep = TT(timestep), tlen = TT(step_length);
    auto q = get_sycl_queue();
    auto mesh = make_mesh(q, nx, ny, dx, dy);
    const size_t nc = nx * ny, nf = mesh->template object_count<MeshComponent::Face>();
    PinBed<T>::z = vec(z, nc);
    SaintVenantConstants<T, Cartesian2DMesh> K(mesh, true);
    State<T> U(T(0), mesh), dUdx(T(0), mesh), dUdy(T(0), mesh), dUdt(T(0), mesh);
    set_state(U, q, mesh, h, u, v, nc);
    SaintVenantFluxes<T, Cartesian2DMesh> F(mesh);

    U.calculate_spatial_derivatives(dUdx, dUdy);
    F.update(U, K, dUdx, dUdy);
    using TDKernel = SaintVenantTemporalDerivativeKernel<T, Cartesian2DMesh>;
    q->submit([&](sycl::handler& cgh) {
      auto kernel = TDKernel(cgh, U, K, dUdx, dUdy, F, dUdt, tnow, tstep);
      cgh.parallel_for(sycl::range<1>(nc), kernel);
    });
    if (ns) {
      CF<T> fns(q, "n_shallow", mesh, vec(ns, nc), true), fnd(q, "n_deep", mesh, vec(nd, nc), true);
      CF<T> fds(q, "d_shallow", mesh, vec(ds, nc), true), fdd(q, "d_deep", mesh, vec(dd, nc), true);
      CF<T> nh(q, "mannings_n", mesh, 0.0f, true), Sf(q, "friction_slope", mesh, 0.0f, true);
      using Kernel = ManningRoughnessSourceKernel<TT, T, Cartesian2DMesh>;
      q->submit([&](sycl::handler& cgh) {
        auto kernel = Kernel(cgh, U, K, fns, fnd, fds, fdd, nh, Sf, dUdt, tstep);
        cgh.parallel_for(sycl::range<1>(nc), kernel);
      });
    }
    auto discharge = [&]() {
      if (!q0) return;
      CF<T> f0(q, "qbdy0", mesh, vec(q0, nc), true), f1(q, "qbdy1", mesh, vec(q1, nc), true);
      using Kernel = DischargeBoundarySourceKernel<T, Cartesian2DMesh>;
      q->submit([&](sycl::handler& cgh) {
        auto kernel = Kernel(cgh, U, K, f0, f1, dUdt, tstep, tnow, tlen);
        cgh.parallel_for(sycl::range<1>(nc), kernel);
      });
    };
    auto head = [&]() {
      if (!hb0) return;
      CF<T> f0(q, "hbdy0", mesh, vec(hb0, nc), true), f1(q, "hbdy1", mesh, vec(hb1, nc), true);
      using Kernel = HeadBoundarySourceKernel<T, Cartesian2DMesh>;
      q->submit([&](sycl::handler& cgh) {
        auto kernel = Kernel(cgh, U, K, f0, f1, dUdt, tstep, tnow, tlen);
        cgh.parallel_for(sycl::range<1>(nc), kernel);
      });
    };
    if (head_first) { head(); discharge(); }
    else { discharge(); head(); }

    T* o = out;
    CF<T>* cells[] = {const_cast<CF<T>*>(&K.dzdx_bed()), const_cast<CF<T>*>(&K.dzdy_bed()),
                      &dUdx.h(), &dUdx.u(), &dUdx.v(), &dUdy.h(), &dUdy.u(), &dUdy.v()};
    for (CF<T>* f : cells) { read(*f, o); o += nc; }
    using FF = FaceField<T, Cartesian2DMesh>;
    FF* faces[] = {&F.h(), &F.u(), &F.v(), &F.z(), F.template get_output_field_ptr<FF>("flux-branch")};
    for (FF* f : faces) { read(*f, o); o += nf; }
    CF<T>* ks[] = {&dUdt.h(), &dUdt.u(), &dUdt.v()};
    for (CF<T>* f : ks) { read(*f, o); o += nc; }
    return 0;
  } catch (const std::exception& e) {
    std::cerr << "ref_pin: " << e.what() << std::endl;
    return -1;
  }
}

// One update_dUdt with the further source and boundary terms. f[] holds the optional per-cell
// arrays (null = term off): 0-3 Manning n_shallow, n_deep, d_shallow, d_deep; 4-5 energy-loss
// fx, fy; 6 infiltration rate (icap, the capacity, is read and written back); 7 the eddy-
// viscosity coefficient mu (eddy mode 1); 8-9 discharge q0, q1; 10-11 stage levels l0, l1.
// iopt: eddy mode (0 off, 1 coefficient field, 2 Smagorinsky with dopt[0], dopt[1]), head_first
// (the stage boundary before the discharge), and the configured order of the momentum terms
// (three codes: 1 roughness, 2 energy loss, 3 eddy viscosity). Infiltration, which touches
// dh/dt only, runs after them. dopt: mu_const, mu_smag, time_now, timestep, step_length.
// out: dh/dt, du/dt, dv/dt.
template <typename T>
int dudt_terms(uint64_t nx, uint64_t ny, double dx, double dy, const T* z, const T* h, const T* u, const T* v,
               const T* const* f, T* icap, const int* iopt, const double* dopt, T* out) {
  try {
    using TT = T;
    const TT tnow = TT(dopt[2]), tstep = TT(dopt[3]), tlen = TT(dopt[4]);
    auto q = get_sycl_queue();
    auto mesh = make_mesh(q, nx, ny, dx, dy);
    const size_t nc = nx * ny;
    PinBed<T>::z = vec(z, nc);
    SaintVenantConstants<T, Cartesian2DMesh> K(mesh, true);
    State<T> U(T(0), mesh), dUdx(T(0), mesh), dUdy(T(0), mesh), dUdt(T(0), mesh);
    set_state(U, q, mesh, h, u, v, nc);
    SaintVenantFluxes<T, Cartesian2DMesh> F(mesh);
    U.calculate_spatial_derivatives(dUdx, dUdy);
    F.update(U, K, dUdx, dUdy);
    using TDKernel = SaintVenantTemporalDerivativeKernel<T, Cartesian2DMesh>;
    q->submit([&](sycl::handler& cgh) {
      auto kernel = TDKernel(cgh, U, K, dUdx, dUdy, F, dUdt, tnow, tstep);
      cgh.parallel_for(sycl::range<1>(nc), kernel);
    });
    auto manning = [&]() {
      if (!f[0]) return;
      CF<T> fns(q, "n_shallow", mesh, vec(f[0], nc), true), fnd(q, "n_deep", mesh, vec(f[1], nc), true);
      CF<T> fds(q, "d_shallow", mesh, vec(f[2], nc), true), fdd(q, "d_deep", mesh, vec(f[3], nc), true);
      CF<T> nh(q, "mannings_n", mesh, 0.0f, true), Sf(q, "friction_slope", mesh, 0.0f, true);
      using Kernel = ManningRoughnessSourceKernel<TT, T, Cartesian2DMesh>;
      q->submit([&](sycl::handler& cgh) {
        auto kernel = Kernel(cgh, U, K, fns, fnd, fds, fdd, nh, Sf, dUdt, tstep);
        cgh.parallel_for(sycl::range<1>(nc), kernel);
      });
    };
    auto eloss = [&]() {
      if (!f[4]) return;
      CF<T> fx(q, "fx", mesh, vec(f[4], nc), true), fy(q, "fy", mesh, vec(f[5], nc), true);
      using Kernel = EnergyLossSourceKernel<TT, T, Cartesian2DMesh>;
      q->submit([&](sycl::handler& cgh) {
        auto kernel = Kernel(cgh, U, K, fx, fy, dUdt, tstep);
        cgh.parallel_for(sycl::range<1>(nc), kernel);
      });
    };
    auto eddy = [&]() {
      if (iopt[0] == 0) return;
      // EddyViscositySourceTerm::apply (EddyViscositySourceTerm.hpp:222-257)
      using SpatialDerivative = SpatialDerivativeOperator<T, Cartesian2DMesh, MeshComponent::Cell, Minmod3<T>>;
      CF<T> d2udx2(q, "d2udx2", mesh, 0.0, true), d2udy2(q, "d2udy2", mesh, 0.0, true);
      CF<T> d2vdx2(q, "d2vdx2", mesh, 0.0, true), d2vdy2(q, "d2vdy2", mesh, 0.0, true);
      SpatialDerivative::template apply<SpatialDerivativeAxis::X>(dUdx.u(), d2udx2);
      SpatialDerivative::template apply<SpatialDerivativeAxis::Y>(dUdy.u(), d2udy2);
      SpatialDerivative::template apply<SpatialDerivativeAxis::X>(dUdx.v(), d2vdx2);
      SpatialDerivative::template apply<SpatialDerivativeAxis::Y>(dUdy.v(), d2vdy2);
      const T mu_const = T(iopt[0] == 2 ? dopt[0] : std::nan("")), mu_smag = T(iopt[0] == 2 ? dopt[1] : std::nan(""));
      CF<T> mu(q, "mu", mesh, iopt[0] == 1 ? vec(f[7], nc) : std::vector<T>(nc, T(0)), true);
      if (!(mu_const != mu_const) && !(mu_smag != mu_smag)) {
        q->submit([&](sycl::handler& cgh) {
          auto kernel = SmagorinskyCoefficientKernel<T, Cartesian2DMesh>(cgh, mu_const, mu_smag, dUdx.u(), dUdy.u(),
                                                                         dUdx.v(), dUdy.v(), mu);
          cgh.parallel_for(sycl::range<1>(nc), kernel);
        });
      }
      using Kernel = EddyViscositySourceKernel<TT, T, Cartesian2DMesh>;
      q->submit([&](sycl::handler& cgh) {
        auto kernel = Kernel(cgh, U, K, mu, d2udx2, d2udy2, d2vdx2, d2vdy2, dUdt, tstep);
        cgh.parallel_for(sycl::range<1>(nc), kernel);
      });
    };
    for (int i = 0; i < 3; ++i) {
      const int t = iopt[2 + i];
      if (t == 1) manning();
      else if (t == 2) eloss();
      else if (t == 3) eddy();
    }
    CF<T> cap(q, "infiltration_capacity", mesh, icap ? vec(icap, nc) : std::vector<T>(nc, T(0)), true);
    if (f[6]) {
      CF<T> rate(q, "infiltration_rate", mesh, vec(f[6], nc), true);
      using Kernel = InfiltrationSourceKernel<TT, T, Cartesian2DMesh>;
      q->submit([&](sycl::handler& cgh) {
        auto kernel = Kernel(cgh, U, K, rate, cap, dUdt, tstep);
        cgh.parallel_for(sycl::range<1>(nc), kernel);
      });
    }
    auto discharge = [&]() {
      if (!f[8]) return;
      CF<T> f0(q, "qbdy0", mesh, vec(f[8], nc), true), f1(q, "qbdy1", mesh, vec(f[9], nc), true);
      using Kernel = DischargeBoundarySourceKernel<T, Cartesian2DMesh>;
      q->submit([&](sycl::handler& cgh) {
        auto kernel = Kernel(cgh, U, K, f0, f1, dUdt, tstep, tnow, tlen);
        cgh.parallel_for(sycl::range<1>(nc), kernel);
      });
    };
    auto stage = [&]() {
      if (!f[10]) return;
      CF<T> f0(q, "hbdy0", mesh, vec(f[10], nc), true), f1(q, "hbdy1", mesh, vec(f[11], nc), true);
      using Kernel = StageBoundarySourceKernel<T, Cartesian2DMesh>;
      q->submit([&](sycl::handler& cgh) {
        auto kernel = Kernel(cgh, U, K, f0, f1, dUdt, double(tstep), double(tnow), double(tlen));
        cgh.parallel_for(sycl::range<1>(nc), kernel);
      });
    };
    if (iopt[1]) { stage(); discharge(); }
    else { discharge(); stage(); }
    T* o = out;
    CF<T>* ks[] = {&dUdt.h(), &dUdt.u(), &dUdt.v()};
    for (CF<T>* k : ks) { read(*k, o); o += nc; }
    if (icap) read(cap, icap);
    return 0;
  } catch (const std::exception& e) {
    std::cerr << "ref_pin: " << e.what() << std::endl;
    return -1;
  }
}

// The cell fields `values[k]` named `names[k]` on an nx x ny mesh of cell size dx, dy with its
// origin at (ox, oy), written by the reference's formatter for a FieldOutputFunction (as
// MultiFieldOutputFile::timed_output does, OutputFile.hpp:195-223): CSVOutput with `delimiter`,
// or RawBinaryOutput when `binary`.
template <typename T>
int write_fields(uint64_t nx, uint64_t ny, double dx, double dy, double ox, double oy, int nfields,
                 const char* const* names, const T* const* values, const char* delimiter, int binary,
                 const char* path) {
  try {
    auto q = get_sycl_queue();
    Config& c = GlobalConfig::instance().mesh;
    auto mesh = make_mesh(q, nx, ny, dx, dy);
    {
      std::ostringstream o;
      o.precision(17);
      o << ox << ", " << oy;
      c.kv["origin"] = o.str();
      mesh = std::make_shared<Cartesian2DMesh>(q, true);
      c.kv.erase("origin");
    }
    const size_t nc = nx * ny;
    std::vector<std::unique_ptr<CF<T>>> fields;
    std::vector<CF<T>*> ptrs;
    for (int k = 0; k < nfields; ++k) {
      fields.emplace_back(new CF<T>(q, names[k], mesh, vec(values[k], nc), true));
      ptrs.push_back(fields.back().get());
    }
    auto of = std::make_shared<FieldOutputFunction<CF<T>>>(ptrs);
    if (binary) {
      RawBinaryOutput(of).output(path);
    } else {
      CSVOutput(of, delimiter).output(path);
    }
    return 0;
  } catch (const std::exception& e) {
    std::cerr << "ref_pin: " << e.what() << std::endl;
    return -1;
  }
}

// A measure's points (times t, values v) as the reference writes them (Measure::output,
// src/Output/Measure.hpp:82-97): CSVOutput over TimeSeriesOutputFunction, whose first column
// "ID" holds the times in the value type. PinSeries stands in for the reference's TimeSeries
// with the two arrays the output function reads.
template <typename TT, typename T>
struct PinSeries {
  using TimeType = TT;
  using ValueType = T;
  struct Array {
    std::vector<T> v;
    const std::vector<T>& host_vector() const { return v; }
  };
  Array t, x;
  const Array& get_time_array() const { return t; }
  const Array& get_value_array() const { return x; }
};
template <typename T>
int write_series(uint64_t n, const double* t, const T* v, const char* name, const char* path) {
  try {
    auto ts = std::make_shared<PinSeries<T, T>>();
    for (uint64_t i = 0; i < n; ++i) {
      ts->t.v.push_back(T(t[i]));
      ts->x.v.push_back(v[i]);
    }
    auto of = std::make_shared<TimeSeriesOutputFunction<PinSeries<T, T>>>(name, ts);
    CSVOutput(of).output(path);
    return 0;
  } catch (const std::exception& e) {
    std::cerr << "ref_pin: " << e.what() << std::endl;
    return -1;
  }
}

// Cartesian2DMesh::get_nearest_object_index<Cell> (Cartesian2DMesh.hpp:179-188) of n locations
// xy (x0, y0, x1, y1, ...) on an nx x ny mesh of cell size dx, dy with its origin at (ox, oy):
// the cell containing each location, nx * ny outside the mesh; and, when loc is not null, the
// cell centres get_object_location<Cell> (x, y per cell) of every cell.
int nearest_cells(uint64_t nx, uint64_t ny, double dx, double dy, double ox, double oy, uint64_t n,
                  const double* xy, uint64_t* out, double* loc) {
  try {
    auto q = get_sycl_queue();
    Config& c = GlobalConfig::instance().mesh;
    make_mesh(q, nx, ny, dx, dy);  // sets the cell count and size
    std::ostringstream o;
    o.precision(17);
    o << ox << ", " << oy;
    c.kv["origin"] = o.str();
    auto mesh = std::make_shared<Cartesian2DMesh>(q, false);
    c.kv.erase("origin");
    for (uint64_t i = 0; i < n; ++i)
      out[i] = mesh->get_nearest_object_index<MeshComponent::Cell>({xy[2 * i], xy[2 * i + 1]});
    if (loc) {
      for (uint64_t i = 0; i < nx * ny; ++i) {
        const std::array<double, 2> p = mesh->get_object_location<MeshComponent::Cell>(i);
        loc[2 * i] = p[0];
        loc[2 * i + 1] = p[1];
      }
    }
    return 0;
  } catch (const std::exception& e) {
    std::cerr << "ref_pin: " << e.what() << std::endl;
    return -1;
  }
}

// SaintVenantState::max_control_number (State.cpp:195-230) of (h, u, v) for `timestep`
template <typename T>
int control_number(uint64_t nx, uint64_t ny, double dx, double dy, const T* h, const T* u, const T* v, double timestep,
                   T* cn) {
  try {
    auto q = get_sycl_queue();
    auto mesh = make_mesh(q, nx, ny, dx, dy);
    State<T> U(T(0), mesh);
    set_state(U, q, mesh, h, u, v, nx * ny);
    *cn = U.max_control_number(timestep);
    return 0;
  } catch (const std::exception& e) {
    std::cerr << "ref_pin: " << e.what() << std::endl;
    return -1;
  }
}

// RungeKuttaSolver::update_y (RungeKutta.hpp:377-388) through the SaintVenantState
// operators: Y = U0, then Y += k_col * (a_col * timestep) for col = 0 .. ncols-1.
template <typename T>
int update_y(uint64_t nx, uint64_t ny, double dx, double dy, const T* u0, const T* k, int ncols, const double* a,
             double timestep, T* y) {
  try {
    auto q = get_sycl_queue();
    auto mesh = make_mesh(q, nx, ny, dx, dy);
    const size_t nc = nx * ny;
    State<T> U0(T(0), mesh), Y(T(0), mesh);
    set_state(U0, q, mesh, u0, u0 + nc, u0 + 2 * nc, nc);
    std::vector<std::unique_ptr<State<T>>> K;
    for (int c = 0; c < ncols; ++c) {
      K.emplace_back(new State<T>(T(0), mesh));
      const T* kc = k + size_t(c) * 3 * nc;
      set_state(*K.back(), q, mesh, kc, kc + nc, kc + 2 * nc, nc);
    }
    Y = U0;
    for (int c = 0; c < ncols; ++c) Y += *K[c] * (a[c] * timestep);
    read(Y.h(), y);
    read(Y.u(), y + nc);
    read(Y.v(), y + 2 * nc);
    return 0;
  } catch (const std::exception& e) {
    std::cerr << "ref_pin: " << e.what() << std::endl;
    return -1;
  }
}

// Problem handed to PinSolver (RungeKuttaSolver constructs its solver itself).
template <typename T>
struct PinProblem {
  uint64_t nx = 0, ny = 0;
  double dx = 1, dy = 1;
  std::vector<T> z, h, u, v;
  bool manning = false;
  T n[4] = {};
  std::vector<double> rain_t, rain_v;  // rain time series knots (m/s); empty: no discharge term
  unsigned head_edges = 0;             // SV_EDGE_* bits of the head strips; 0: no head term
  T head_value = 0;
  bool head_first = false;
  uint64_t timesteps = 0;              // do_timestep calls (accepted + repeated)
};
template <typename T>
PinProblem<T>* g_problem = nullptr;

// TimeSeries::at with ts_linterp (src/Input/TimeSeries.cpp:26-47), last segment extrapolated
double series_at(const std::vector<double>& t, const std::vector<double>& v, double time) {
  size_t i1 = 1;
  while (i1 < t.size() && !(t[i1] > time)) ++i1;
  if (i1 >= t.size()) i1 = t.size() - 1;
  const size_t i0 = i1 - 1;
  const double dvdt = (v[i1] - v[i0]) / (t[i1] - t[i0]);
  return v[i0] + dvdt * (time - t[i0]);
}

// Stand-in for SaintVenantSolver<T, T, Cartesian2DMesh> with its interface to RungeKuttaSolver.
template <typename T>
class PinSolver {
 public:
  using TimeType = T;
  using ValueType = T;
  using MeshType = Cartesian2DMesh;
  using StateT = SaintVenantState<T, Cartesian2DMesh>;

  PinSolver(const std::shared_ptr<sycl::queue>& q, const size_t& nstates, const std::shared_ptr<TimeParameters<T>>& tp)
      : q_(q), P_(*g_problem<T>) {
    mesh_ = make_mesh(q, P_.nx, P_.ny, P_.dx, P_.dy);
    const size_t nc = P_.nx * P_.ny;
    PinBed<T>::z = P_.z;
    K_ = std::make_shared<SaintVenantConstants<T, Cartesian2DMesh>>(mesh_, true);
    for (size_t i = 0; i < nstates; ++i) {
      U_.push_back(std::make_shared<StateT>(T(0), mesh_));
      dUdt_.push_back(std::make_shared<StateT>(T(0), mesh_));
    }
    set_state(*U_[0], q, mesh_, P_.h.data(), P_.u.data(), P_.v.data(), nc);
    dUdx_ = std::make_shared<StateT>(T(0), mesh_);
    dUdy_ = std::make_shared<StateT>(T(0), mesh_);
    F_ = std::make_shared<SaintVenantFluxes<T, Cartesian2DMesh>>(mesh_);
    const char* names[4] = {"n_shallow", "n_deep", "d_shallow", "d_deep"};
    for (int i = 0; i < 4; ++i) man_.emplace_back(q, names[i], mesh_, P_.n[i], true);
    nh_ = std::make_shared<CF<T>>(q, "mannings_n", mesh_, 0.0f, true);
    Sf_ = std::make_shared<CF<T>>(q, "friction_slope", mesh_, 0.0f, true);
    q0_ = std::make_shared<CF<T>>(q, "qbdy0", mesh_, 0.0f, true);
    q1_ = std::make_shared<CF<T>>(q, "qbdy1", mesh_, 0.0f, true);
    const T nan = std::numeric_limits<T>::quiet_NaN();
    hb0_ = std::make_shared<CF<T>>(q, "hbdy0", mesh_, nan, true);
    hb1_ = std::make_shared<CF<T>>(q, "hbdy1", mesh_, nan, true);
  }

  // SaintVenantSolver::update_dUdt (Solver.cpp:73-114)
  void update_dUdt(const size_t& state_no, const T& time_now, const T& timestep) {
    StateT& U = *U_.at(state_no);
    StateT& D = *dUdt_.at(state_no);
    U.calculate_spatial_derivatives(*dUdx_, *dUdy_);
    F_->update(U, *K_, *dUdx_, *dUdy_);
    const size_t nc = mesh_->template object_count<MeshComponent::Cell>();
    using TDKernel = SaintVenantTemporalDerivativeKernel<T, Cartesian2DMesh>;
    q_->submit([&](sycl::handler& cgh) {
      auto kernel = TDKernel(cgh, U, *K_, *dUdx_, *dUdy_, *F_, D, time_now, timestep);
      cgh.parallel_for(sycl::range<1>(nc), kernel);
    });
    if (P_.manning) {
      using Kernel = ManningRoughnessSourceKernel<T, T, Cartesian2DMesh>;
      q_->submit([&](sycl::handler& cgh) {
        auto kernel = Kernel(cgh, U, *K_, man_[0], man_[1], man_[2], man_[3], *nh_, *Sf_, D, timestep);
        cgh.parallel_for(sycl::range<1>(nc), kernel);
      });
    }
    const T tlen = TimeType(step_length_);
    auto discharge = [&]() {
      if (P_.rain_t.empty()) return;
      using Kernel = DischargeBoundarySourceKernel<T, Cartesian2DMesh>;
      q_->submit([&](sycl::handler& cgh) {
        auto kernel = Kernel(cgh, U, *K_, *q0_, *q1_, D, timestep, time_now, tlen);
        cgh.parallel_for(sycl::range<1>(nc), kernel);
      });
    };
    auto head = [&]() {
      if (!P_.head_edges) return;
      using Kernel = HeadBoundarySourceKernel<T, Cartesian2DMesh>;
      q_->submit([&](sycl::handler& cgh) {
        auto kernel = Kernel(cgh, U, *K_, *hb0_, *hb1_, D, timestep, time_now, tlen);
        cgh.parallel_for(sycl::range<1>(nc), kernel);
      });
    };
    if (P_.head_first) { head(); discharge(); }
    else { discharge(); head(); }
  }

  // DischargeBoundarySourceTerm / HeadBoundarySourceTerm::start_new_step
  // (DischargeBoundarySourceTerm.hpp:114-146, HeadBoundarySourceTerm.hpp:114-146): clear the
  // values (BoundarySourceTerm::clear_values) and add the rain at t and t + L everywhere; set
  // the head values on the edge strips.
  void start_new_step(const T& time_now, const std::shared_ptr<TimeParameters<T>>& tp) {
    step_length_ = tp->step_duration();
    if (!P_.rain_t.empty()) {
      *q0_ = 0.0;
      *q1_ = 0.0;
      *q0_ += T(series_at(P_.rain_t, P_.rain_v, time_now));
      *q1_ += T(series_at(P_.rain_t, P_.rain_v, time_now + step_length_));
    }
    if (P_.head_edges) {
      *hb0_ = 0.0;
      *hb1_ = 0.0;
      hb0_->move_to_host();
      hb1_->move_to_host();
      std::vector<T>& a = const_cast<std::vector<T>&>(hb0_->data().host_vector());
      std::vector<T>& b = const_cast<std::vector<T>&>(hb1_->data().host_vector());
      for (size_t i = 0; i < a.size(); ++i) {
        const size_t x = i % P_.nx, y = i / P_.nx;
        const bool sel = ((P_.head_edges & 1u) && x == 0) || ((P_.head_edges & 2u) && x == P_.nx - 1) ||
                         ((P_.head_edges & 4u) && y == 0) || ((P_.head_edges & 8u) && y == P_.ny - 1);
        if (sel) { a[i] = P_.head_value; b[i] = P_.head_value; }
      }
      hb0_->move_to_device();
      hb1_->move_to_device();
    }
  }
  void end_of_step(const T&) {}

  StateT& state(const size_t& i = 0) { return *U_.at(i); }
  StateT& dUdt(const size_t& i) { return *dUdt_.at(i); }
  ValueType control_number(const size_t& state_no, const TimeType& timestep) {
    ++P_.timesteps;
    return U_.at(state_no)->max_control_number(timestep);
  }

 private:
  std::shared_ptr<sycl::queue> q_;
  PinProblem<T>& P_;
  std::shared_ptr<Cartesian2DMesh> mesh_;
  std::shared_ptr<SaintVenantConstants<T, Cartesian2DMesh>> K_;
  std::vector<std::shared_ptr<StateT>> U_, dUdt_;
  std::shared_ptr<StateT> dUdx_, dUdy_;
  std::shared_ptr<SaintVenantFluxes<T, Cartesian2DMesh>> F_;
  std::vector<CF<T>> man_;
  std::shared_ptr<CF<T>> nh_, Sf_, q0_, q1_, hb0_, hb1_;
  T step_length_ = T(60);
};

template <typename T>
struct PinScheme : public RungeKuttaSolver<PinSolver<T>> {
  using RungeKuttaSolver<PinSolver<T>>::RungeKuttaSolver;
  PinSolver<T>& solver() { return *this->solver_; }
};

// RungeKuttaSolver<...>::solve over [start, end] with the named tableau `rk`.
template <typename T>
int solve(uint64_t nx, uint64_t ny, double dx, double dy, const T* z, const T* h, const T* u, const T* v,
          const double* manning, const double* rain_t, const double* rain_v, int nrain, unsigned head_edges,
          double head_value, int head_first, const char* rk, double start, double end, double step_length,
          double initial_dt, T* out, uint64_t* timesteps) {
  try {
    const size_t nc = nx * ny;
    PinProblem<T> P;
    P.nx = nx; P.ny = ny; P.dx = dx; P.dy = dy;
    P.z = vec(z, nc); P.h = vec(h, nc); P.u = vec(u, nc); P.v = vec(v, nc);
    P.manning = manning != nullptr;
    for (int i = 0; i < 4; ++i) P.n[i] = manning ? T(manning[i]) : T(0);
    for (int i = 0; i < nrain; ++i) { P.rain_t.push_back(rain_t[i]); P.rain_v.push_back(rain_v[i]); }
    P.head_edges = head_edges;
    P.head_value = T(head_value);
    P.head_first = head_first != 0;
    g_problem<T> = &P;
    Config conf;
    std::ostringstream s;
    s.precision(17);
    auto put = [&](const char* k, double x) { s.str(""); s << x; conf.kv[k] = s.str(); };
    put("start time", start);
    put("end time", end);
    put("step duration seconds", step_length);
    put("initial timestep seconds", initial_dt);
    auto tp = std::make_shared<TimeParameters<T>>(conf);
    PinScheme<T> scheme(tp, std::string(rk), get_sycl_queue());
    scheme.solve();
    read(scheme.solver().state().h(), out);
    read(scheme.solver().state().u(), out + nc);
    read(scheme.solver().state().v(), out + 2 * nc);
    *timesteps = P.timesteps;
    g_problem<T> = nullptr;
    return 0;
  } catch (const std::exception& e) {
    std::cerr << "ref_pin: " << e.what() << std::endl;
    return -1;
  }
}

}  // namespace

extern "C" {
int refpin_solve_f64(uint64_t nx, uint64_t ny, double dx, double dy, const double* z, const double* h, const double* u,
                     const double* v, const double* manning, const double* rain_t, const double* rain_v, int nrain,
                     unsigned head_edges, double head_value, int head_first, const char* rk, double start, double end,
                     double step_length, double initial_dt, double* out, uint64_t* timesteps) {
  return solve<double>(nx, ny, dx, dy, z, h, u, v, manning, rain_t, rain_v, nrain, head_edges, head_value, head_first,
                       rk, start, end, step_length, initial_dt, out, timesteps);
}
int refpin_solve_f32(uint64_t nx, uint64_t ny, double dx, double dy, const float* z, const float* h, const float* u,
                     const float* v, const double* manning, const double* rain_t, const double* rain_v, int nrain,
                     unsigned head_edges, double head_value, int head_first, const char* rk, double start, double end,
                     double step_length, double initial_dt, float* out, uint64_t* timesteps) {
  return solve<float>(nx, ny, dx, dy, z, h, u, v, manning, rain_t, rain_v, nrain, head_edges, head_value, head_first,
                      rk, start, end, step_length, initial_dt, out, timesteps);
}
int refpin_dudt_f64(uint64_t nx, uint64_t ny, double dx, double dy, const double* z, const double* h, const double* u,
                    const double* v, const double* ns, const double* nd, const double* ds, const double* dd,
                    const double* q0, const double* q1, const double* hb0, const double* hb1, int head_first,
                    double time_now, double timestep, double step_length, double* out) {
  return dudt<double>(nx, ny, dx, dy, z, h, u, v, ns, nd, ds, dd, q0, q1, hb0, hb1, head_first, time_now, timestep,
                      step_length, out);
}
int refpin_dudt_f32(uint64_t nx, uint64_t ny, double dx, double dy, const float* z, const float* h, const float* u,
                    const float* v, const float* ns, const float* nd, const float* ds, const float* dd, const float* q0,
                    const float* q1, const float* hb0, const float* hb1, int head_first, double time_now,
                    double timestep, double step_length, float* out) {
  return dudt<float>(nx, ny, dx, dy, z, h, u, v, ns, nd, ds, dd, q0, q1, hb0, hb1, head_first, time_now, timestep,
                     step_length, out);
}
int refpin_dudt_terms_f64(uint64_t nx, uint64_t ny, double dx, double dy, const double* z, const double* h,
                          const double* u, const double* v, const double* const* f, double* icap, const int* iopt,
                          const double* dopt, double* out) {
  return dudt_terms<double>(nx, ny, dx, dy, z, h, u, v, f, icap, iopt, dopt, out);
}
int refpin_dudt_terms_f32(uint64_t nx, uint64_t ny, double dx, double dy, const float* z, const float* h,
                          const float* u, const float* v, const float* const* f, float* icap, const int* iopt,
                          const double* dopt, float* out) {
  return dudt_terms<float>(nx, ny, dx, dy, z, h, u, v, f, icap, iopt, dopt, out);
}
int refpin_write_fields_f64(uint64_t nx, uint64_t ny, double dx, double dy, double ox, double oy, int nfields,
                            const char* const* names, const double* const* values, const char* delimiter, int binary,
                            const char* path) {
  return write_fields<double>(nx, ny, dx, dy, ox, oy, nfields, names, values, delimiter, binary, path);
}
int refpin_write_fields_f32(uint64_t nx, uint64_t ny, double dx, double dy, double ox, double oy, int nfields,
                            const char* const* names, const float* const* values, const char* delimiter, int binary,
                            const char* path) {
  return write_fields<float>(nx, ny, dx, dy, ox, oy, nfields, names, values, delimiter, binary, path);
}
int refpin_write_series_f64(uint64_t n, const double* t, const double* v, const char* name, const char* path) {
  return write_series<double>(n, t, v, name, path);
}
int refpin_write_series_f32(uint64_t n, const double* t, const float* v, const char* name, const char* path) {
  return write_series<float>(n, t, v, name, path);
}
// TimeParameters::num_steps (TimeParameters.cpp:40-58) for start, end and step duration in
// seconds, TimeType double
int refpin_num_steps(double start, double end, double step, uint64_t* n) {
  try {
    Config conf;
    std::ostringstream s;
    s.precision(17);
    auto put = [&](const char* k, double x) { s.str(""); s << x; conf.kv[k] = s.str(); };
    put("start time", start);
    put("end time", end);
    put("step duration seconds", step);
    TimeParameters<double> tp(conf);
    *n = tp.num_steps();
    return 0;
  } catch (const std::exception& e) {
    std::cerr << "ref_pin: " << e.what() << std::endl;
    return -1;
  }
}
int refpin_nearest_cells(uint64_t nx, uint64_t ny, double dx, double dy, double ox, double oy, uint64_t n,
                         const double* xy, uint64_t* out, double* loc) {
  return nearest_cells(nx, ny, dx, dy, ox, oy, n, xy, out, loc);
}
int refpin_control_number_f64(uint64_t nx, uint64_t ny, double dx, double dy, const double* h, const double* u,
                              const double* v, double timestep, double* cn) {
  return control_number<double>(nx, ny, dx, dy, h, u, v, timestep, cn);
}
int refpin_control_number_f32(uint64_t nx, uint64_t ny, double dx, double dy, const float* h, const float* u,
                              const float* v, double timestep, float* cn) {
  return control_number<float>(nx, ny, dx, dy, h, u, v, timestep, cn);
}
int refpin_update_y_f64(uint64_t nx, uint64_t ny, double dx, double dy, const double* u0, const double* k, int ncols,
                        const double* a, double timestep, double* y) {
  return update_y<double>(nx, ny, dx, dy, u0, k, ncols, a, timestep, y);
}
int refpin_update_y_f32(uint64_t nx, uint64_t ny, double dx, double dy, const float* u0, const float* k, int ncols,
                        const double* a, double timestep, float* y) {
  return update_y<float>(nx, ny, dx, dy, u0, k, ncols, a, timestep, y);
}
}
