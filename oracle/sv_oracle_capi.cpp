// sv_oracle_capi.cpp -- TEST INFRASTRUCTURE: C-ABI over the CPU oracle (sv_oracle.hpp).
//
// The entry points mirror include/sv.h one for one (prefix svo_ instead of sv_), so a
// test can run the same call sequence against the CUDA library and against this oracle.
// Precision SV_F64 instantiates Solver<double,double> (the reference templates at
// T = TT = double); SV_F32 instantiates Solver<float,float>, the precision of the shipped
// reference binary (src/mfcm.cpp:13-16).
#include <cstdio>
#include <exception>
#include <string>

#include "../include/sv.h"
#include "sv_oracle.hpp"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {
thread_local std::string g_err;

int fail(const std::exception& e) {
  g_err = e.what();
  return SV_E_ARG;
}

svo::Params to_params(const sv_params* p) {
  svo::Params q;
  q.rk_method = p->rk_method;
  q.cn_target = p->cn_target;
  q.step_duration = p->step_duration;
  q.initial_dt = p->initial_dt;
  q.max_dt = p->max_dt;
  q.rain_mode = p->rain_mode;
  q.manning = p->manning;
  q.head_first = p->head_first;
  q.eloss_first = (p->flags & SV_FLAG_ELOSS_FIRST) ? 1 : 0;
  return q;
}
}  // namespace

extern "C" {

int svo_create(const sv_mesh_desc* mesh, const sv_params* params, void** out) {
  try {
    if (!mesh || !params || !out) throw std::runtime_error("null argument");
    if (mesh->nx == 0 || mesh->ny == 0) throw std::runtime_error("empty mesh");
    svo::Mesh m;
    m.nx = mesh->nx; m.ny = mesh->ny; m.dx = std::fabs(mesh->dx); m.dy = std::fabs(mesh->dy);
    svo::Params q = to_params(params);
    svo::SolverBase* s = nullptr;
    if (params->precision == SV_F64) s = new svo::Solver<double, double>(m, q);
    else s = new svo::Solver<float, float>(m, q);
    s->set_track_tallies(!(params->flags & SV_FLAG_NO_TALLIES));
    *out = s;
    return 0;
  } catch (const std::exception& e) { return fail(e); }
}

void svo_destroy(void* h) { delete static_cast<svo::SolverBase*>(h); }

int svo_set_field(void* h, int id, const double* src, uint64_t n) {
  try { static_cast<svo::SolverBase*>(h)->set_field(id, src, n); return 0; }
  catch (const std::exception& e) { return fail(e); }
}
int svo_get_field(void* h, int id, double* dst, uint64_t n) {
  try { static_cast<svo::SolverBase*>(h)->get_field(id, dst, n); return 0; }
  catch (const std::exception& e) { return fail(e); }
}
int svo_set_manning(void* h, double a, double b, double c, double d) {
  static_cast<svo::SolverBase*>(h)->set_manning(a, b, c, d);
  return 0;
}
int svo_set_eddy_viscosity(void* h, int mode, double mu, double mc, double ms) {
  try { static_cast<svo::SolverBase*>(h)->set_eddy(mode, mu, mc, ms); return 0; }
  catch (const std::exception& e) { return fail(e); }
}
int svo_set_source_order(void* h, const int* terms, int n) {
  try { static_cast<svo::SolverBase*>(h)->set_source_order(terms, n); return 0; }
  catch (const std::exception& e) { return fail(e); }
}
int svo_set_forcing(void* h, const sv_forcing* f) {
  svo::Forcing g;
  g.rain_kind = f->rain_kind; g.rain_q0 = f->rain_q0; g.rain_q1 = f->rain_q1;
  g.head_kind = f->head_kind; g.head_edges = f->head_edges; g.head_h0 = f->head_h0; g.head_h1 = f->head_h1;
  static_cast<svo::SolverBase*>(h)->set_forcing(g);
  return 0;
}
int svo_set_dt(void* h, double dt) { static_cast<svo::SolverBase*>(h)->set_dt(dt); return 0; }
int svo_get_dt(void* h, double* dt) { *dt = static_cast<svo::SolverBase*>(h)->get_dt(); return 0; }
int svo_eval_dudt(void* h, int state_no, double t_sub, double dt) {
  try { static_cast<svo::SolverBase*>(h)->update_dUdt(size_t(state_no), t_sub, dt); return 0; }
  catch (const std::exception& e) { return fail(e); }
}
int svo_do_timestep(void* h, double t_local, double dt, double* cn, int* repeat, double* new_dt) {
  static_cast<svo::SolverBase*>(h)->do_timestep(t_local, dt, cn, repeat, new_dt);
  return 0;
}
int svo_accept(void* h) { static_cast<svo::SolverBase*>(h)->accept(); return 0; }
int svo_advance(void* h, sv_stats* out) {
  svo::Stats st;
  static_cast<svo::SolverBase*>(h)->step(&st);
  if (out) {
    out->accepted = st.accepted; out->repeated = st.repeated; out->volume = st.volume;
    out->rain_in = st.rain_in; out->outflow = st.outflow; out->wall_in = st.wall_in;
  }
  return 0;
}
int svo_get_stats(void* h, sv_stats* out) {
  svo::Stats st = static_cast<svo::SolverBase*>(h)->stats();
  out->accepted = st.accepted; out->repeated = st.repeated; out->volume = st.volume;
  out->rain_in = st.rain_in; out->outflow = st.outflow; out->wall_in = st.wall_in;
  return 0;
}
int svo_set_stats(void* h, const sv_stats* in) {
  svo::Stats st{};
  st.accepted = in->accepted; st.repeated = in->repeated; st.rain_in = in->rain_in; st.outflow = in->outflow;
  st.wall_in = in->wall_in;
  static_cast<svo::SolverBase*>(h)->set_stats(st);
  return 0;
}
int svo_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}
// x^(4/3) as used by the FP64 Manning term, exposed for its accuracy test
double svo_pow43(double x) { return sv_math::pow43(x); }
double svo_minmod3(double ul, double dxl, double uc, double dxr, double ur) {
  return svo::minmod3<double>(ul, dxl, uc, dxr, ur);
}
float svo_minmod3f(float ul, double dxl, float uc, double dxr, float ur) {
  return svo::minmod3<float>(ul, dxl, uc, dxr, ur);
}
const char* svo_last_error(void) { return g_err.c_str(); }

}  // extern "C"
