// sv_kernels.cuh -- kernels of the Saint-Venant RK time step on sm_100a.
//
//  stage_kernel   one launch per RK stage. A CTA owns a TX x TY tile of cells, stages the
//                 tile plus a 2-cell halo of (h, u, v, z) in shared memory, computes the
//                 Minmod3 slopes of every cell of the tile plus a 1-cell ring, the fluxes of
//                 every face of the tile, then per cell dU/dt (flux divergence, depth-slope,
//                 limited bed slope, zflux), Manning friction, rainfall and outflow, and the
//                 Runge-Kutta combination. Faces and slopes never leave the SM. The last
//                 stage also reduces the CFL quantity and the FP64 volume per CTA.
//  finalize_kernel  one CTA: fixed-order reduction of the per-CTA partials, the control
//                 number, and the dt controller (accept / repeat / new dt / end-of-step
//                 trimming) in FP64, so a whole step runs without a host round trip.
//  debug kernels  the same per-face / per-cell functions over global arrays, one reference
//                 kernel each, for per-function parity tests.
#pragma once
#include "sv_device.cuh"

namespace svk {
using namespace svd;

// Device-resident controller state of one solver (FP64 times, TT = double).
struct Ctl {
  double t_local;   // time since the start of the step
  double dt;        // current timestep
  double cn;        // control number of the last timestep
  double new_dt;    // dt suggested by the last timestep
  int cur;          // parity of the state buffer that holds U_[0]
  int done;         // 1: the step is complete (auto mode) -- all stage kernels exit
  int repeat;       // last timestep rejected
  int error;        // sticky error code (SV_E_NONFINITE ...)
  unsigned long long accepted, repeated;            // running totals
  unsigned long long step_accepted, step_repeated;  // in the current step
  double rain_in, outflow;      // running tallies over accepted timesteps
  double wall_in;               // running tally of the flow through the mesh-edge faces
  double volume;                // volume of U_[0] after the last accepted timestep
  double pend_rain, pend_out, pend_vol;  // tallies of the last timestep, applied on accept
  double pend_wall;
  long long budget;             // > 0: timesteps left before the loop pauses (done = 2)
};

// Per-step boundary values, kept in device memory so captured graphs stay valid when
// start_new_step changes them (DischargeBoundarySourceTerm.hpp:114-146,
// HeadBoundarySourceTerm.hpp:114-146).
struct DevForcing {
  int rain_kind;        // SV_RAIN_*
  int head_kind;        // SV_HEAD_*
  unsigned head_edges;  // SV_EDGE_* bits
  int pad;
  double rq0, rq1;      // uniform / pattern-scaled rain values at the start / end of the step
  double hh0, hh1;      // head targets at the start / end of the step
};

enum StageMode : int {
  M_FIRST = 1,    // stage 0: input is U_[0]
  M_LAST = 2,     // last stage: writes U_[N] and the CFL / volume partials
  M_ACC = 4,      // diagonal tableau: running accumulator instead of stored k's
  M_STOREK = 8,   // store k_s for later stages (non-diagonal tableaux)
  M_TALLY = 16,   // rain / outflow partials
  M_DEBUGK = 32,  // debug: write k_s only (no RK combination)
};

template <typename T> struct StageParams {
  int nx, ny;
  double dx, dy, L;
  double cell_area;
  T* S[2][3];            // state parity buffers: S[cur] = U_[0], S[cur^1] = acc / U_[N]
  const T* Yin[3];       // stage input (ignored on the first stage)
  T* Yout[3];            // Y_{s+1} (not on the last stage)
  T* Kout[3];            // k_s (M_STOREK / M_DEBUGK)
  const T* Kin[4][3];    // stored k_j, j < s (M_STOREK)
  const T* z;
  const T* zx; const T* zy;   // bed slopes dz/dx, dz/dy (Constants.cpp:39-40), precomputed
  const double* zdat;         // FP32-with-datum mode: per datum tile FP64 datum (z = datum + z_off)
  int dtiles_x;               // datum tiles per row
  const T* man_p[4];     // per-cell n_shallow, n_deep, d_shallow, d_deep, or nullptr
  T man_s[4];            // uniform values where man_p is nullptr
  const DevForcing* fc;  // per-step boundary values
  const T* q0p; const T* q1p; const T* pat;
  const T* hb0p; const T* hb1p;
  const T* irate; T* icap;   // infiltration rate (m/s) and remaining capacity (m), or nullptr
  const T* efx; const T* efy;  // energy-loss coefficients fx/m, fy/m, or nullptr
  T* hc[2];              // FP32: per-cell compensation of the depth update (state parity), or nullptr
  int manning, rain_mode, head_first;
  int eloss_first;       // energy loss applied before roughness (configuration order)
  int stage, nstages, mode;
  double c_s;            // c of this stage: t_sub = t_local + c_s * dt
  double a_next[4];      // a(s+2, j+1), j = 0..s: coefficients of Y_{s+1}
  double b[4];           // b_1..b_N
  Ctl* ctl;
  double* part;          // per-CTA partials (see part_* offsets)
  long long nblk;
  // eddy viscosity (run by the kernels compiled with it): 0 off, 1 constant coefficient
  // (eddy_mup per cell, else eddy_mu), 2 Smagorinsky (eddy_c + eddy_s * area * |strain|)
  int eddy;
  T eddy_mu, eddy_c, eddy_s;
  const T* eddy_mup;
  // the momentum source terms in configuration order, 2 bits per slot: 1 roughness,
  // 2 energy loss, 3 eddy viscosity (each adds to du/dt and dv/dt, so the order sets the
  // rounding); used by the kernels compiled with eddy viscosity
  int term_order;
  // column-sweep strips split by kind (see strip_flags_kernel): the interior strips run the
  // interior kernel, the others the general one; null lists: every strip runs the general one
  const int* istrips;
  const int* bstrips;
  int n_istrips, n_bstrips;
  // two-cells-per-lane variants: pairs of adjacent interior strips (the first strip of each);
  // istrips then lists the interior strips left out of a pair
  const int* ipairs;
  int n_ipairs;
  // split schedule: the stage input's slopes dh/dx, du/dx, dv/dx, dh/dy, du/dy, dv/dy as
  // written by slopes_kernel (read by the stage kernel instead of computing them), or null
  T* pslp[6];
};

// partial layout: [0, nblk) cn max, [nblk, 2nblk) cn min, [2nblk, 3nblk) volume,
// then rain[s] at (3 + 3s) nblk, outflow[s] at (4 + 3s) nblk, wall flow[s] at (5 + 3s) nblk.
__host__ __device__ inline long long part_count(long long nblk, int nstages) { return (3 + 3LL * nstages) * nblk; }

template <typename T> __device__ __forceinline__ T ld(const T* p, long long i) { return __ldg(p + i); }
// Loads of the state, stage and accumulator buffers. A launch that writes and later reads them
// itself (the persistent batch kernel, COH) must use coherent loads, ordered by its phase
// fences; every other launch only reads what earlier launches wrote, through the read-only path.
template <bool COH, typename T> __device__ __forceinline__ T ldst(const T* p, long long i) {
  if constexpr (COH) return p[i];
  return __ldg(p + i);
}

// Datum tiles of the FP32-with-datum mode: 32 x 8 cells, each with an FP64 datum; the stored
// bed is the FP32 offset from its tile's datum.
constexpr int kDatumTX = 32, kDatumTY = 8;
__host__ __device__ inline long long datum_tile(int gx, int gy, int dtiles_x) {
  return (long long)(gy / kDatumTY) * dtiles_x + gx / kDatumTX;
}
// FP32 with tile datums: the beds of a face's two cells, (ax, ay) below or left of (bx, by),
// in the frame of the lower cell's datum tile: b's offset moved by the exact FP64 datum
// difference and rounded once, a's unchanged.
template <typename T>
__device__ __forceinline__ void face_frame(const StageParams<T>& P, CellV<T>& a, CellV<T>& b, int ax, int ay, int bx,
                                           int by) {
  const long long ta = datum_tile(ax, ay, P.dtiles_x), tb = datum_tile(bx, by, P.dtiles_x);
  if (ta != tb) b.z = T(double(b.z) + (P.zdat[tb] - P.zdat[ta]));
}

// Bed of cell (gx, gy) in the frame of datum tile `ref`: the stored value itself, or, for a
// cell of another datum tile, its offset moved by the FP64 datum difference and rounded once.
template <typename T>
__device__ __forceinline__ T load_bed(const T* z, const double* zdat, int dtiles_x, long long g, int gx, int gy,
                                      long long ref) {
  const T zo = __ldg(z + g);
  if (!zdat) return zo;
  const long long t = datum_tile(gx, gy, dtiles_x);
  if (t == ref) return zo;
  return T(double(zo) + (__ldg(zdat + t) - __ldg(zdat + ref)));
}

// NaN-propagating max/min for the CFL reduction
__device__ __forceinline__ double nmax(double a, double b) { return (a != a || b != b) ? (a + b) : (a > b ? a : b); }
__device__ __forceinline__ double nmin(double a, double b) { return (a != a || b != b) ? (a + b) : (a < b ? a : b); }
__device__ __forceinline__ float nmax(float a, float b) { return (a != a || b != b) ? (a + b) : (a > b ? a : b); }
__device__ __forceinline__ float nmin(float a, float b) { return (a != a || b != b) ? (a + b) : (a < b ? a : b); }

template <int NT> __device__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < NT / 32; ++i) r += red[i];
  }
  return r;
}
template <int NT> __device__ double block_max(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v = nmax(v, __shfl_down_sync(0xffffffffu, v, o));
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double r = v;
  if (threadIdx.x == 0) {
    r = red[0];
    for (int i = 1; i < NT / 32; ++i) r = nmax(r, red[i]);
  }
  return r;
}
template <int NT> __device__ double block_min(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v = nmin(v, __shfl_down_sync(0xffffffffu, v, o));
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double r = v;
  if (threadIdx.x == 0) {
    r = red[0];
    for (int i = 1; i < NT / 32; ++i) r = nmin(r, red[i]);
  }
  return r;
}

template <typename T> __device__ __forceinline__ Div<T> mkdiv(double d);
template <> __device__ __forceinline__ Div<double> mkdiv<double>(double d) { return make_div(d); }
template <> __device__ __forceinline__ Div<float> mkdiv<float>(double d) { return make_divf(float(d)); }
template <typename DV> struct MkDivX;
template <> struct MkDivX<DivD> { __device__ static DivD make(double d) { return make_div(d); } };
template <> struct MkDivX<DivP2> { __device__ static DivP2 make(double d) { return DivP2{1.0 / d}; } };
template <> struct MkDivX<DivF> { __device__ static DivF make(double d) { return make_divf(float(d)); } };

// Per-cell dU/dt of one stage (TemporalDerivativeKernel.cpp:53-98, then the source terms
// and boundaries in configuration order, Solver.cpp:97-113). fw/fe/fs/fn are the four face
// fluxes; returns the rain rate added, the depth rate removed by the head assignment and the
// depth rate that entered through mesh-edge faces (the reference's walls pass flow through
// their one-sided branches; taken before any boundary assignment).
template <typename T, typename CC, bool EDDY = false, bool EDGE = true>
__device__ __forceinline__ void cell_dudt(const StageParams<T>& P, const DevForcing& fc, const CC& c,
                                          long long g, int gx,
                                          int gy, T h, T u, T v, T dhdx, T dhdy, T dzdx, T dzdy,
                                          const FaceF<T>& fw, const FaceF<T>& fe, const FaceF<T>& fs,
                                          const FaceF<T>& fn, T& kh, T& ku, T& kv, double& rain,
                                          double& removed, double& wall, T* n_out, T* sf_out,
                                          const EddyIn<T>* ed = nullptr) {
  T dhdt = c.divx(fw.h - fe.h) + c.divy(fs.h - fn.h);
  T dudt = c.divx(fw.u - fe.u) + c.divy(fs.u - fn.u);
  T dvdt = c.divx(fw.v - fe.v) + c.divy(fs.v - fn.v);
  dudt = dudt + dhdx * T(-kG);
  dvdt = dvdt + dhdy * T(-kG);
  T hdx = c.divx(h), hdy = c.divy(h);
  if (sfabs(dzdx) > hdx) dzdx = (dzdx > T(0)) ? hdx : ((dzdx < T(0)) ? -hdx : c.divx(ssign(dzdx) * h));
  if (sfabs(dzdy) > hdy) dzdy = (dzdy > T(0)) ? hdy : ((dzdy < T(0)) ? -hdy : c.divy(ssign(dzdy) * h));
  T dudt_bed = T(-kG) * dzdx;
  T dvdt_bed = T(-kG) * dzdy;
  dudt = dudt + c.divx(fw.z - fe.z);
  dvdt = dvdt + c.divy(fs.z - fn.z);
  dudt = dudt + dudt_bed;
  dvdt = dvdt + dvdt_bed;
  // source terms in configuration order (Solver.cpp:98-104): roughness and energy loss both
  // add to du/dt, dv/dt, so only their relative order changes the rounding
  auto do_manning = [&]() {
    if (!P.manning) return;
    T ns = P.man_p[0] ? ld(P.man_p[0], g) : P.man_s[0];
    T nd = P.man_p[1] ? (P.man_p[1] == P.man_p[0] ? ns : ld(P.man_p[1], g)) : P.man_s[1];
    T ds = P.man_p[2] ? ld(P.man_p[2], g) : P.man_s[2];
    T dd = P.man_p[3] ? ld(P.man_p[3], g) : P.man_s[3];
    manning_apply<T>(h, u, v, ns, nd, ds, dd, c, dudt, dvdt, n_out, sf_out);
  };
  auto do_eloss = [&]() {
    if (P.efx) energy_loss_apply<T>(h, u, v, ld(P.efx, g), ld(P.efy, g), c, dudt, dvdt);
  };
  if constexpr (!EDDY) {
    if (P.eloss_first) { do_eloss(); do_manning(); }
    else { do_manning(); do_eloss(); }
  } else {
    // each term's increments depend on the cell's state only; they are added in the
    // configured order
    T fu1 = T(0), fv1 = T(0), fu2 = T(0), fv2 = T(0), fu3 = T(0), fv3 = T(0);
    bool on1 = false, on2 = false, on3 = false;
    if (P.manning) {
      T ns = P.man_p[0] ? ld(P.man_p[0], g) : P.man_s[0];
      T nd = P.man_p[1] ? (P.man_p[1] == P.man_p[0] ? ns : ld(P.man_p[1], g)) : P.man_s[1];
      T ds = P.man_p[2] ? ld(P.man_p[2], g) : P.man_s[2];
      T dd = P.man_p[3] ? ld(P.man_p[3], g) : P.man_s[3];
      on1 = manning_term<T>(h, u, v, ns, nd, ds, dd, c, fu1, fv1, n_out, sf_out);
    }
    if (P.efx) on2 = energy_loss_term<T>(h, u, v, ld(P.efx, g), ld(P.efy, g), c, fu2, fv2);
    if (P.eddy) {
      const T mu = P.eddy == 2 ? smagorinsky_mu<T>(P.eddy_c, P.eddy_s, T(P.cell_area), *ed)
                               : (P.eddy_mup ? ld(P.eddy_mup, g) : P.eddy_mu);
      on3 = eddy_term<T>(h, u, v, mu, *ed, c, fu3, fv3);
    }
#pragma unroll
    for (int s = 0; s < 3; ++s) {
      const int t = (P.term_order >> (2 * s)) & 3;
      if (t == 1 && on1) { dudt = dudt + fu1; dvdt = dvdt + fv1; }
      else if (t == 2 && on2) { dudt = dudt + fu2; dvdt = dvdt + fv2; }
      else if (t == 3 && on3) { dudt = dudt + fu3; dvdt = dvdt + fv3; }
    }
  }
  if (P.irate) {  // infiltration (InfiltrationSourceTerm.cpp:43-62), capacity consumed in place
    T cap = P.icap[g];
    T dh = infiltration_depth<T>(h, ld(P.irate, g), cap, c);
    dhdt = dhdt - c.divdt(dh);
    P.icap[g] = cap - dh;
  }
  rain = 0.0;
  removed = 0.0;
  wall = 0.0;
  if constexpr (EDGE) {  // cells away from the mesh edge have no wall faces
    if (gx == 0) wall += double(c.divx(fw.h));
    if (gx == P.nx - 1) wall -= double(c.divx(fe.h));
    if (gy == 0) wall += double(c.divy(fs.h));
    if (gy == P.ny - 1) wall -= double(c.divy(fn.h));
  }
  // head boundary target values for this cell (NaN = not selected); a stage boundary
  // (StageBoundarySourceTerm.cpp:48-52) gives water levels, from which the bed is subtracted
  bool head_sel = false;
  T h0 = T(0), h1 = T(0);
  const int hk = fc.head_kind;
  if (hk == 1 || hk == 3) {
    if constexpr (EDGE) {  // edge strips: never a cell away from the mesh edge
      head_sel = ((fc.head_edges & 1u) && gx == 0) || ((fc.head_edges & 2u) && gx == P.nx - 1) ||
                 ((fc.head_edges & 4u) && gy == 0) || ((fc.head_edges & 8u) && gy == P.ny - 1);
      h0 = T(fc.hh0); h1 = T(fc.hh1);
    }
  } else if (hk == 2 || hk == 4) {
    h0 = ld(P.hb0p, g); h1 = ld(P.hb1p, g);
    head_sel = true;
  }
  if (head_sel && hk >= 3) {
    if (P.zdat) {  // absolute bed = FP64 datum + FP32 offset; levels minus bed in FP64
      const double zb = P.zdat[datum_tile(gx, gy, P.dtiles_x)] + double(ld(P.z, g));
      h0 = T(double(h0) - zb); h1 = T(double(h1) - zb);
    } else {
      const T zb = ld(P.z, g);
      h0 = h0 - zb; h1 = h1 - zb;
    }
  }
  if (head_sel && !(h0 == h0 && h1 == h1)) head_sel = false;  // NaN = not selected
  auto do_rain = [&]() {
    if (fc.rain_kind == 0) return;
    T q0, q1;
    if (fc.rain_kind == 1) { q0 = T(fc.rq0); q1 = T(fc.rq1); }
    else if (fc.rain_kind == 2) { q0 = ld(P.q0p, g); q1 = ld(P.q1p, g); }
    else { T pp = ld(P.pat, g); q0 = pp * T(fc.rq0); q1 = pp * T(fc.rq1); }
    bool applied;
    T dh = discharge_rate<T>(q0, q1, h, c, applied);
    if (applied) { dhdt = dhdt + dh; rain = double(dh); }
  };
  auto do_head = [&]() {
    if (!head_sel) return;
    T target = head_target<T>(h0, h1, c);
    T before = dhdt;
    dhdt = c.divdt(target - h);
    removed = double(before) - double(dhdt);
  };
  if (P.head_first) { do_head(); do_rain(); }
  else { do_rain(); do_head(); }
  kh = dhdt; ku = dudt; kv = dvdt;
}

// One cell of one stage after its four face fluxes are known: dU/dt, then the Runge-Kutta
// combination (RungeKutta.hpp:377-388) and, on the last stage, the CFL quantity and volume.
template <typename T, typename CC, bool EDDY = false, bool EDGE = true, bool COH = false>
__device__ __forceinline__ void finish_cell(const StageParams<T>& P, const DevForcing& fc, const CC& c,
                                            long long g, int gx, int gy, T h, T u, T v, T dhdx, T dhdy, T dzdx,
                                            T dzdy, const FaceF<T>& fw, const FaceF<T>& fe, const FaceF<T>& fs,
                                            const FaceF<T>& fn, bool first, bool last, int cur, double dt_d,
                                            double& rain, double& removed, double& walls, T& xcfl,
                                            T& xcfl_min, double& vol, const EddyIn<T>* ed = nullptr) {
  T kh, ku, kv;
  double r_, o_, w_;
  cell_dudt<T, CC, EDDY, EDGE>(P, fc, c, g, gx, gy, h, u, v, dhdx, dhdy, dzdx, dzdy, fw, fe, fs, fn, kh, ku, kv, r_,
                               o_, w_, (T*)nullptr, (T*)nullptr, ed);
  rain += r_;
  removed += o_;
  walls += w_;
  if (P.mode & (M_STOREK | M_DEBUGK)) {
    P.Kout[0][g] = kh; P.Kout[1][g] = ku; P.Kout[2][g] = kv;
  }
  if (P.mode & M_DEBUGK) return;
  const int st = P.stage;
  T* A[3] = {P.S[cur ^ 1][0], P.S[cur ^ 1][1], P.S[cur ^ 1][2]};
  const T* U0[3] = {P.S[cur][0], P.S[cur][1], P.S[cur][2]};
  T k[3] = {kh, ku, kv};
  T out[3];
  if (P.mode & M_ACC) {
    // diagonal tableau: Y_{s+1} = U0 + k_s*a and acc += k_s*b, in the reference's
    // left-to-right order (RungeKutta.hpp:377-388); the skipped zero-coefficient terms
    // k_j*0 (j < s) can only contribute a NaN, which happens exactly when some earlier
    // k_j is not finite, i.e. when acc is not finite while U0 is.
    const T cB = T(P.b[st] * dt_d);
    // FP32 (hc set): the accumulator holds the increment sum_s k_s cB_s, added to U0 once at
    // the last stage; the depth takes it with a per-cell compensation carried across
    // timesteps. Rounding a small, nearly uniform increment (steady rain) onto the depth at
    // every stage otherwise biases the FP32 volume by ~1e-4 over thousands of timesteps.
    const bool incr = sizeof(T) == 4 && P.hc[0] != nullptr;
    T u0v[3], accv[3];
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      u0v[f] = first ? (f == 0 ? h : (f == 1 ? u : v)) : ldst<COH>(U0[f], g);
      accv[f] = first ? (incr ? T(0) : u0v[f]) : ldst<COH>(A[f], g);
    }
    if (!last) {
      const T cA = T(P.a_next[st] * dt_d);
#pragma unroll
      for (int f = 0; f < 3; ++f) {
        T y = u0v[f] + k[f] * cA;
        // FP32 leaves this out: a non-finite accumulator reaches U_N at the last stage anyway
        if constexpr (sizeof(T) == 8)
          if (!first && finite_(u0v[f]) && !finite_(accv[f])) y = Lim<T>::nan();
        P.Yout[f][g] = y;
      }
    }
    if (!incr) {
#pragma unroll
      for (int f = 0; f < 3; ++f) {
        out[f] = accv[f] + k[f] * cB;
        A[f][g] = out[f];
      }
    } else {
#pragma unroll
      for (int f = 0; f < 3; ++f) {
        const T d = accv[f] + k[f] * cB;  // increment sum so far
        if (!last) {
          A[f][g] = d;
          out[f] = d;
        } else if (f == 0) {  // U_N.h = U0.h + d with the carried compensation (Neumaier)
          const T y = d + ldst<COH>(P.hc[cur], g);
          const T t = u0v[0] + y;
          P.hc[cur ^ 1][g] = (sfabs(u0v[0]) >= sfabs(y)) ? (u0v[0] - t) + y : (y - t) + u0v[0];
          out[0] = t;
          A[0][g] = t;
        } else {
          out[f] = u0v[f] + d;
          A[f][g] = out[f];
        }
      }
    }
  } else {
    // general tableau: Y_{s+1} = ((U0 + k_0 c_0) + k_1 c_1) + ... with stored k_j
    T u0v[3];
#pragma unroll
    for (int f = 0; f < 3; ++f) u0v[f] = first ? (f == 0 ? h : (f == 1 ? u : v)) : ldst<COH>(U0[f], g);
    const double* coef = last ? P.b : P.a_next;
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      T y = u0v[f];
      for (int j = 0; j < st; ++j) y = y + ldst<COH>(P.Kin[j][f], g) * T(coef[j] * dt_d);
      y = y + k[f] * T(coef[st] * dt_d);
      out[f] = y;
      if (last) A[f][g] = y;
      else P.Yout[f][g] = y;
    }
  }
  if (last) {
    // SaintVenantState::max_control_number (State.cpp:204-228) on U_[N]: per cell
    // x = (|u|+c)/dx + (|v|+c)/dy; cn = max(dt*x) = dt*max(x) (rounding is monotone)
    T hh = sfmax(out[0], T(0));
    T cc = ssqrt(T(kG) * hh);
    T xx = c.divx(sfabs(out[1]) + cc) + c.divy(sfabs(out[2]) + cc);
    xcfl = nmax(xcfl, xx);  // a max or min of T values is exact in T
    xcfl_min = nmin(xcfl_min, xx);
    vol += double(out[0]) * P.cell_area;
  }
}

template <typename T, int TX, int TY>
struct StageSmem {
  static constexpr int RX = TX + 4, RY = TY + 4;  // values with a 2-cell halo
  static constexpr int SX = TX + 2, SY = TY + 2;  // slopes with a 1-cell ring
  T val[4][RY][RX];
  T slp[8][SY][SX];
  T fxf[4][TY][TX + 1];
  T fyf[4][TY + 1][TX];
  double red[TX * TY / 32];
};

// One TX x TY tile of one stage: bx, by = tile coordinates, blk = partial-sum slot.
template <typename T, int TX, int TY, bool P2, bool EDDY, bool PRE = false>
__device__ __forceinline__ void stage_tile(const StageParams<T>& P, int bx, int by, long long blk,
                                           StageSmem<T, TX, TY>& s) {
  using DX = DivX<T, P2>;
  using SM = StageSmem<T, TX, TY>;
  constexpr int NT = TX * TY;

  const Ctl* ctl = P.ctl;
  if (ctl->done) return;
  const int cur = ctl->cur;
  const double dt_d = ctl->dt;
  const double tsub = ctl->t_local + P.c_s * dt_d;

  const int tid = threadIdx.x;
  const int x0 = bx * TX, y0 = by * TY;
  const int nx = P.nx, ny = P.ny;
  const bool first = P.mode & M_FIRST;
  const T* Yh = first ? P.S[cur][0] : P.Yin[0];
  const T* Yu = first ? P.S[cur][1] : P.Yin[1];
  const T* Yv = first ? P.S[cur][2] : P.Yin[2];

  // phase 1: tile + 2-cell halo of h, u, v, z (clamped at the mesh edge; the clamped
  // copies are never used because edge faces and edge slopes use the cell itself)
  const long long zref = P.zdat ? datum_tile(x0, y0, P.dtiles_x) : 0;
  for (int i = tid; i < SM::RX * SM::RY; i += NT) {
    int lx = i % SM::RX, ly = i / SM::RX;
    int gx = min(max(x0 - 2 + lx, 0), nx - 1);
    int gy = min(max(y0 - 2 + ly, 0), ny - 1);
    long long g = (long long)gy * nx + gx;
    s.val[0][ly][lx] = ld(Yh, g);
    s.val[1][ly][lx] = ld(Yu, g);
    s.val[2][ly][lx] = ld(Yv, g);
    s.val[3][ly][lx] = load_bed(P.z, P.zdat, P.dtiles_x, g, gx, gy, zref);
  }
  __syncthreads();

  const DX divx = MkDivX<DX>::make(P.dx), divy = MkDivX<DX>::make(P.dy);
  // phase 2: Minmod3 slopes of h, u, v (State.cpp:176-193) on the tile + ring; the bed
  // slopes (Constants.cpp:39-40) are precomputed once per bed and loaded
  for (int i = tid; i < SM::SX * SM::SY; i += NT) {
    int sx = i % SM::SX, sy = i / SM::SX;
    if ((sx == 0 || sx == SM::SX - 1) && (sy == 0 || sy == SM::SY - 1)) continue;  // unused corners
    int gx = x0 - 1 + sx, gy = y0 - 1 + sy;
    if (gx < 0 || gx >= nx || gy < 0 || gy >= ny) continue;
    int lx = sx + 1, ly = sy + 1;
    bool hasW = gx > 0, hasE = gx < nx - 1, hasN = gy < ny - 1, hasS = gy > 0;
    long long g = (long long)gy * nx + gx;
    s.slp[3][sy][sx] = ld(P.zx, g);
    s.slp[7][sy][sx] = ld(P.zy, g);
    if constexpr (PRE) {  // split schedule: slopes from the slopes pass
#pragma unroll
      for (int f = 0; f < 3; ++f) {
        s.slp[f][sy][sx] = ld(P.pslp[f], g);
        s.slp[4 + f][sy][sx] = ld(P.pslp[3 + f], g);
      }
    } else {
#pragma unroll
      for (int f = 0; f < 3; ++f) {
        s.slp[f][sy][sx] = minmod3<T>(s.val[f][ly][lx - 1], hasW, s.val[f][ly][lx], hasE, s.val[f][ly][lx + 1], divx);
        // Y axis: north (row + 1) is the left neighbour, south the right
        s.slp[4 + f][sy][sx] =
            minmod3<T>(s.val[f][ly + 1][lx], hasN, s.val[f][ly][lx], hasS, s.val[f][ly - 1][lx], divy);
      }
    }
  }
  __syncthreads();

  auto cellv = [&](int gx, int gy) {
    int sx = gx - (x0 - 1), sy = gy - (y0 - 1);
    int lx = sx + 1, ly = sy + 1;
    CellV<T> c;
    c.h = s.val[0][ly][lx]; c.u = s.val[1][ly][lx]; c.v = s.val[2][ly][lx]; c.z = s.val[3][ly][lx];
    c.dhdx = s.slp[0][sy][sx]; c.dudx = s.slp[1][sy][sx]; c.dvdx = s.slp[2][sy][sx]; c.dzdx = s.slp[3][sy][sx];
    c.dhdy = s.slp[4][sy][sx]; c.dudy = s.slp[5][sy][sx]; c.dvdy = s.slp[6][sy][sx]; c.dzdy = s.slp[7][sy][sx];
    return c;
  };
  // phase 3: face fluxes (Fluxes.cpp:44-65)
  const T hdx = T(0.5) * T(P.dx), hdy = T(0.5) * T(P.dy);
  for (int i = tid; i < (TX + 1) * TY; i += NT) {
    int fx = i % (TX + 1), fy = i / (TX + 1);
    int gfx = x0 + fx, gy = y0 + fy;
    if (gy >= ny || gfx > nx) continue;
    int edge = gfx == 0 ? -1 : (gfx == nx ? 1 : 0);
    int gl = edge == -1 ? 0 : gfx - 1;
    int gr = edge == 1 ? nx - 1 : gfx;
    FaceF<T> F;
    face_flux<T, 0>(cellv(gl, gy), cellv(gr, gy), edge, hdx, divx, F);
    s.fxf[0][fy][fx] = F.h; s.fxf[1][fy][fx] = F.u; s.fxf[2][fy][fx] = F.v; s.fxf[3][fy][fx] = F.z;
  }
  for (int i = tid; i < TX * (TY + 1); i += NT) {
    int fx = i % TX, fy = i / TX;
    int gx = x0 + fx, gfy = y0 + fy;
    if (gx >= nx || gfy > ny) continue;
    int edge = gfy == 0 ? -1 : (gfy == ny ? 1 : 0);
    int gl = edge == -1 ? 0 : gfy - 1;
    int gr = edge == 1 ? ny - 1 : gfy;
    FaceF<T> F;
    face_flux<T, 1>(cellv(gx, gl), cellv(gx, gr), edge, hdy, divy, F);
    s.fyf[0][fy][fx] = F.h; s.fyf[1][fy][fx] = F.u; s.fyf[2][fy][fx] = F.v; s.fyf[3][fy][fx] = F.z;
  }
  __syncthreads();

  // phase 4: per cell
  const int tx = tid % TX, ty = tid / TX;
  const int gx = x0 + tx, gy = y0 + ty;
  const bool valid = gx < nx && gy < ny;
  double rain = 0.0, removed = 0.0, walls = 0.0, vol = 0.0;
  T xcfl = T(0), xcfl_min = T(1.0 / 0.0);
  const bool last = P.mode & M_LAST;
  if (valid) {
    const long long g = (long long)gy * nx + gx;
    CellCtx<T, DX> c;
    c.divx = divx; c.divy = divy;
    c.divdt = mkdiv<T>(dt_d);
    c.divL = mkdiv<T>(P.L);
    c.dt = T(dt_d); c.dt_d = dt_d; c.tsub_d = tsub;
    c.manning = P.manning; c.rain_mode = P.rain_mode; c.head_first = P.head_first;
    const int sx = tx + 1, sy = ty + 1, lx = tx + 2, ly = ty + 2;
    const T h = s.val[0][ly][lx], u = s.val[1][ly][lx], v = s.val[2][ly][lx];
    FaceF<T> fw{s.fxf[0][ty][tx], s.fxf[1][ty][tx], s.fxf[2][ty][tx], s.fxf[3][ty][tx]};
    FaceF<T> fe{s.fxf[0][ty][tx + 1], s.fxf[1][ty][tx + 1], s.fxf[2][ty][tx + 1], s.fxf[3][ty][tx + 1]};
    FaceF<T> fs{s.fyf[0][ty][tx], s.fyf[1][ty][tx], s.fyf[2][ty][tx], s.fyf[3][ty][tx]};
    FaceF<T> fn{s.fyf[0][ty + 1][tx], s.fyf[1][ty + 1][tx], s.fyf[2][ty + 1][tx], s.fyf[3][ty + 1][tx]};
    const DevForcing fc = *P.fc;
    EddyIn<T> ed{};
    if constexpr (EDDY) {
      if (P.eddy) {  // second derivatives from the slopes of the tile + ring
        const bool hasW = gx > 0, hasE = gx < nx - 1, hasN = gy < ny - 1, hasS = gy > 0;
        ed.ux = s.slp[1][sy][sx]; ed.uy = s.slp[5][sy][sx]; ed.vx = s.slp[2][sy][sx]; ed.vy = s.slp[6][sy][sx];
        ed.uxx = minmod3<T>(s.slp[1][sy][sx - 1], hasW, ed.ux, hasE, s.slp[1][sy][sx + 1], divx);
        ed.vxx = minmod3<T>(s.slp[2][sy][sx - 1], hasW, ed.vx, hasE, s.slp[2][sy][sx + 1], divx);
        ed.uyy = minmod3<T>(s.slp[5][sy + 1][sx], hasN, ed.uy, hasS, s.slp[5][sy - 1][sx], divy);
        ed.vyy = minmod3<T>(s.slp[6][sy + 1][sx], hasN, ed.vy, hasS, s.slp[6][sy - 1][sx], divy);
      }
    }
    finish_cell<T, CellCtx<T, DX>, EDDY>(P, fc, c, g, gx, gy, h, u, v, s.slp[0][sy][sx], s.slp[4][sy][sx],
                                         s.slp[3][sy][sx], s.slp[7][sy][sx], fw, fe, fs, fn, first, last, cur, dt_d,
                                         rain, removed, walls, xcfl, xcfl_min, vol, &ed);
  }
  if (last && !(P.mode & M_DEBUGK)) {
    double mx = block_max<NT>(double(xcfl), s.red);
    double mn = block_min<NT>(double(xcfl_min), s.red);
    double vs = block_sum<NT>(vol, s.red);
    if (tid == 0) {
      P.part[blk] = mx;
      P.part[P.nblk + blk] = mn;
      P.part[2 * P.nblk + blk] = vs;
    }
  }
  if (P.mode & M_TALLY) {
    double rs = block_sum<NT>(rain, s.red);
    double os = block_sum<NT>(removed, s.red);
    double ws = block_sum<NT>(walls, s.red);
    if (tid == 0) {
      P.part[(3 + 3LL * P.stage) * P.nblk + blk] = rs;
      P.part[(4 + 3LL * P.stage) * P.nblk + blk] = os;
      P.part[(5 + 3LL * P.stage) * P.nblk + blk] = ws;
    }
  }
}

template <typename T, int TX, int TY, int MINB, bool P2, bool EDDY, bool PRE = false>
__global__ void __launch_bounds__(TX * TY, MINB) stage_kernel(const StageParams<T> P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  auto& s = *reinterpret_cast<StageSmem<T, TX, TY>*>(smem_raw);
  stage_tile<T, TX, TY, P2, EDDY, PRE>(P, blockIdx.x, blockIdx.y, (long long)blockIdx.y * gridDim.x + blockIdx.x, s);
}

// Split schedule, first pass: the Minmod3 slopes of the stage input (State.cpp:176-193), one
// thread per cell, into P.pslp; the stage kernel that follows reads them instead of forming
// them from its tile.
template <typename T, bool P2>
__global__ void __launch_bounds__(256) slopes_kernel(const StageParams<T> P) {
  using DX = DivX<T, P2>;
  const Ctl* ctl = P.ctl;
  if (ctl->done) return;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int nx = P.nx, ny = P.ny;
  if (i >= (long long)nx * ny) return;
  const int cur = ctl->cur;
  const bool first = P.mode & M_FIRST;
  const int gx = int(i % nx), gy = int(i / nx);
  const bool hasW = gx > 0, hasE = gx < nx - 1, hasN = gy < ny - 1, hasS = gy > 0;
  const DX divx = MkDivX<DX>::make(P.dx), divy = MkDivX<DX>::make(P.dy);
#pragma unroll
  for (int f = 0; f < 3; ++f) {
    const T* a = first ? P.S[cur][f] : P.Yin[f];
    const T c = ld(a, i);
    const T l = hasW ? ld(a, i - 1) : c, r = hasE ? ld(a, i + 1) : c;
    P.pslp[f][i] = minmod3<T>(l, hasW, c, hasE, r, divx);
    // Y axis: north (row + 1) is the left neighbour, south the right
    const T n = hasN ? ld(a, i + nx) : c, so = hasS ? ld(a, i - nx) : c;
    P.pslp[3 + f][i] = minmod3<T>(n, hasN, c, hasS, so, divy);
  }
}

// Batched stage: one launch covers every tile of every instance of a batch. tile_start has
// ninst + 1 entries (prefix sums of the instances' tile counts); each CTA finds its instance,
// copies that instance's parameters to shared memory and runs the same tile body. Instances
// whose step is finished (their controller's done flag) return at once.
template <typename T, int TX, int TY, int MINB, bool P2, bool EDDY>
__global__ void __launch_bounds__(TX * TY, MINB)
    stage_batch_kernel(const StageParams<T>* __restrict__ Ps, const long long* __restrict__ tile_start, int ninst) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  auto& s = *reinterpret_cast<StageSmem<T, TX, TY>*>(smem_raw);
  __shared__ StageParams<T> Psh;
  __shared__ int inst_sh;
  const long long tile = blockIdx.x;
  if (threadIdx.x == 0) {
    int lo = 0, hi = ninst - 1;  // last instance with tile_start[i] <= tile
    while (lo < hi) {
      int mid = (lo + hi + 1) / 2;
      if (tile_start[mid] <= tile) lo = mid;
      else hi = mid - 1;
    }
    inst_sh = lo;
    Psh = Ps[lo];
  }
  __syncthreads();
  const long long local = tile - tile_start[inst_sh];
  const int tiles_x = (Psh.nx + TX - 1) / TX;
  stage_tile<T, TX, TY, P2, EDDY>(Psh, int(local % tiles_x), int(local / tiles_x), local, s);
}

// ---------------------------------------------------------------------------------------
// Column-sweep stage kernel. One warp owns a strip of 32 columns (28 output columns plus a
// 2-column halo on each side) and marches down TY output rows. Each lane holds its column's
// last three rows of (h, u, v, z, dz/dx, dz/dy) and two rows of slopes in registers; x
// neighbours come from warp shuffles, y neighbours from the rolling window. Every face
// flux and every difference quotient is computed once and reused by both cells / both
// slopes that need it, and there is no block-level barrier. The arithmetic per face and
// per cell is the same function as in the tiled kernel.
// ---------------------------------------------------------------------------------------
constexpr unsigned kFull = 0xffffffffu;
template <typename T> __device__ __forceinline__ T up1(T v) { return __shfl_up_sync(kFull, v, 1); }
template <typename T> __device__ __forceinline__ T dn1(T v) { return __shfl_down_sync(kFull, v, 1); }

// The sweeps form slopes with svd::minmod3q (sv_device.cuh): Minmod3 from difference
// quotients, its sign and NaN tests on the integer pipe.
//
// Two-sided Minmod3 of the FP32 interior sweeps: for finite quotients the reference's nested
// pair minmods (Minmod3.hpp:66-80) reduce to sign * min(|2 qL|, |2 qR|, |qC / 2|) when the
// three agree in sign and zero otherwise (up to the sign of a zero result). The NaN rules
// only matter for a non-finite state, as for the dropped tangential terms.
__device__ __forceinline__ float minmod3_finite(float qL, float qR, float qC) {
  const float a = 2.0f * qL, b = 2.0f * qR, c = 0.5f * qC;
  const int ia = __float_as_int(a), ib = __float_as_int(b), ic = __float_as_int(c);
  const float m = fminf(fminf(fabsf(a), fabsf(b)), fabsf(c));
  return ((ia ^ ib) | (ia ^ ic)) >= 0 ? __int_as_float(__float_as_int(m) | (ia & 0x80000000)) : 0.0f;
}
// the interior sweeps' two-sided slope: exact reference rules in FP64, the finite form in FP32
template <typename T> __device__ __forceinline__ T slope2s(T qL, T qR, T qC) {
  if constexpr (sizeof(T) == 4) return minmod3_finite(qL, qR, qC);
  return minmod3q<T>(qL, true, qR, true, qC);
}

template <typename T> struct RowV { T h, u, v, z, zx, zy; };
template <typename T> struct SlopeV { T hx, ux, vx, hy, uy, vy; };

template <typename T>
__device__ __forceinline__ CellV<T> mkcell(const RowV<T>& r, const SlopeV<T>& s) {
  CellV<T> c;
  c.h = r.h; c.u = r.u; c.v = r.v; c.z = r.z;
  c.dhdx = s.hx; c.dudx = s.ux; c.dvdx = s.vx; c.dzdx = r.zx;
  c.dhdy = s.hy; c.dudy = s.uy; c.dvdy = s.vy; c.dzdy = r.zy;
  return c;
}
template <typename T> __device__ __forceinline__ CellV<T> shfl_cell_up(const CellV<T>& a) {
  CellV<T> c;
  c.h = up1(a.h); c.u = up1(a.u); c.v = up1(a.v); c.z = up1(a.z);
  c.dhdx = up1(a.dhdx); c.dudx = up1(a.dudx); c.dvdx = up1(a.dvdx); c.dzdx = up1(a.dzdx);
  c.dhdy = up1(a.dhdy); c.dudy = up1(a.dudy); c.dvdy = up1(a.dvdy); c.dzdy = up1(a.dzdy);
  return c;
}
template <typename T> __device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFull, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = nmax(v, __shfl_down_sync(kFull, v, o));
  return v;
}
__device__ __forceinline__ double warp_min(double v) {
  for (int o = 16; o > 0; o >>= 1) v = nmin(v, __shfl_down_sync(kFull, v, o));
  return v;
}

constexpr int kSweepOut = 28;  // output columns per warp
// Rows the column sweep prefetches into L1 ahead of use: the window fields of row k+1+0 and
// the per-cell fields of output row k-2+3 at iteration k, one iteration ahead. A warp marches
// its rows in order, so without these hints each row's loads wait a full memory latency with
// only one row in flight. One iteration (about 4 us per row at 28 warps per SM) covers the
// latency; prefetching further ahead kept more lines in flight than L1 holds (about 12 KB per
// warp at 3 and 2 rows ahead), and the stages ran 1.5 % (FP32) and 4 % (FP64) slower.
constexpr int kSweepPfWindow = 0, kSweepPfCell = 3;
__device__ __forceinline__ void prefetch_l1(const void* p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }

// Prefetch plan of the interior sweeps. A warp's row of one field is 32 consecutive values of
// an interior strip (columns gx0 .. gx0+31, all inside the mesh): at most two 128-byte lines
// in FP32 and three in FP64. The plan gives each lane kPfSlots (field, line) pairs of the
// fields the stage reads -- the window fields (stage input, bed, bed slopes) first, then the
// per-cell fields -- so that a row ahead costs kPfSlots prefetch instructions per warp instead
// of one per field with its address arithmetic. Pairs beyond 32 * kPfSlots are not prefetched.
constexpr int kPfSlots = 2;
template <typename T> struct PfPlan {
  const T* p[kPfSlots];  // the lane's line in row 0 of its field, or null
  int d[kPfSlots];       // rows ahead of the loop row: the window's or the per-cell fields'
  __device__ __forceinline__ void init(const StageParams<T>& P, const DevForcing& fc, const T* Yh, const T* Yu,
                                       const T* Yv, bool first, int cur, int gx0, int lane) {
    constexpr int kLines = sizeof(T) == 4 ? 2 : 3;
    constexpr int kLineCols = 128 / int(sizeof(T));
    int fi[kPfSlots];
#pragma unroll
    for (int s = 0; s < kPfSlots; ++s) {
      fi[s] = (lane + 32 * s) / kLines;
      p[s] = nullptr;
      d[s] = fi[s] < 6 ? 1 + kSweepPfWindow : kSweepPfCell - 2;
    }
    int n = 0;
    auto add = [&](const T* f) {
#pragma unroll
      for (int s = 0; s < kPfSlots; ++s)
        if (fi[s] == n) p[s] = f;
      ++n;
    };
    add(Yh); add(Yu); add(Yv); add(P.z); add(P.zx); add(P.zy);
    if (!first) {
      for (int f = 0; f < 3; ++f) { add(P.S[cur][f]); add(P.S[cur ^ 1][f]); }
    }
    if (P.manning) {
      for (int f = 0; f < 4; ++f) {
        const T* m = P.man_p[f];
        bool dup = false;
        for (int e = 0; e < f; ++e) dup = dup || (P.man_p[e] == m);
        if (m && !dup) add(m);
      }
    }
    if (P.irate) { add(P.irate); add(P.icap); }
    if (P.efx) { add(P.efx); add(P.efy); }
    if (fc.rain_kind == 3) add(P.pat);
    if (fc.rain_kind == 2) { add(P.q0p); add(P.q1p); }
    if (fc.head_kind == 2) { add(P.hb0p); add(P.hb1p); }
#pragma unroll
    for (int s = 0; s < kPfSlots; ++s)
      if (p[s]) p[s] += gx0 + min(((lane + 32 * s) % kLines) * kLineCols, 31);
  }
  // the rows k + d of every slot, clamped into the mesh
  __device__ __forceinline__ void rows(int k, int nx, int ny) const {
#pragma unroll
    for (int s = 0; s < kPfSlots; ++s)
      if (p[s]) prefetch_l1(p[s] + (long long)min(max(k + d[s], 0), ny - 1) * nx);
  }
};

// One warp's strip `gw` (row-major over strips of kSweepOut columns x TY rows) of one
// solver's stage. Called by the single-solver kernel (P in parameter space) and by the
// batched kernel (P in shared memory).
template <typename T, int TY, bool P2, bool EDDY, bool COH = false>
__device__ __forceinline__ void sweep_strip(const StageParams<T>& P, long long gw) {
  using DX = DivX<T, P2>;
  const Ctl* ctl = P.ctl;
  const int nx = P.nx, ny = P.ny;
  const int tiles_x = (nx + kSweepOut - 1) / kSweepOut;
  const int lane = threadIdx.x;
  const int tile_x = int(gw % tiles_x), tile_y = int(gw / tiles_x);
  const int gx = tile_x * kSweepOut - 2 + lane;
  const int gxc = min(max(gx, 0), nx - 1);
  const bool out_lane = lane >= 2 && lane < 2 + kSweepOut && gx < nx;
  const bool wface_lane = lane >= 2 && lane <= 2 + kSweepOut && gx <= nx;
  const bool hasW = gx > 0, hasE = gx < nx - 1;
  const int y0 = tile_y * TY;

  const int cur = ctl->cur;
  const double dt_d = ctl->dt;
  const double tsub = ctl->t_local + P.c_s * dt_d;
  const bool first = P.mode & M_FIRST, last = P.mode & M_LAST;
  const T* Yh = first ? P.S[cur][0] : P.Yin[0];
  const T* Yu = first ? P.S[cur][1] : P.Yin[1];
  const T* Yv = first ? P.S[cur][2] : P.Yin[2];
  const DX divx = MkDivX<DX>::make(P.dx), divy = MkDivX<DX>::make(P.dy);
  const T hdx = T(0.5) * T(P.dx), hdy = T(0.5) * T(P.dy);
  CellCtx<T, DX> c;
  c.divx = divx; c.divy = divy;
  c.divdt = mkdiv<T>(dt_d);
  c.divL = mkdiv<T>(P.L);
  c.dt = T(dt_d); c.dt_d = dt_d; c.tsub_d = tsub;
  c.manning = P.manning; c.rain_mode = P.rain_mode; c.head_first = P.head_first;
  const DevForcing fc = *P.fc;

  // FP32 with tile datums: the window keeps each cell's raw bed offset; a face whose two
  // cells lie in different datum tiles is evaluated in its lower cell's frame (face_frame),
  // the same whichever strip computes it, so the flux out of one cell is the flux into the
  // other and the volume is conserved across strip boundaries
  auto load_row = [&](int gy) {
    const int r = min(max(gy, 0), ny - 1);
    const long long g = (long long)r * nx + gxc;
    RowV<T> v;
    v.h = ldst<COH>(Yh, g); v.u = ldst<COH>(Yu, g); v.v = ldst<COH>(Yv, g);
    v.z = ld(P.z, g);
    v.zx = ld(P.zx, g); v.zy = ld(P.zy, g);
    return v;
  };

  RowV<T> Rm{}, R0{}, Rp{};   // rows k-2, k-1, k
  SlopeV<T> Sm{}, S0{};       // slopes of rows k-2, k-1
  T Smm_uy = T(0), Smm_vy = T(0);  // y slopes of u, v of row k-3 (eddy viscosity)
  T fyA[3] = {}, fyB[3] = {};  // (U[k-1]-U[k-2])/dy, (U[k]-U[k-1])/dy
  FaceF<T> FS{}, FN{};
  double rain = 0.0, removed = 0.0, walls = 0.0, vol = 0.0;
  T xcfl = T(0), xmin = T(1.0 / 0.0);

  // L1 prefetch of rows ahead (addresses clamped into the mesh, like the loads)
  auto prefetch_rows = [&](int k) {
    {
      const int r = min(max(k + 1 + kSweepPfWindow, 0), ny - 1);
      const long long g = (long long)r * nx + gxc;
      prefetch_l1(Yh + g); prefetch_l1(Yu + g); prefetch_l1(Yv + g);
      prefetch_l1(P.z + g); prefetch_l1(P.zx + g); prefetch_l1(P.zy + g);
    }
    const int r = min(max(k - 2 + kSweepPfCell, 0), ny - 1);
    const long long g = (long long)r * nx + gxc;
    if (!first) {
      for (int f = 0; f < 3; ++f) { prefetch_l1(P.S[cur][f] + g); prefetch_l1(P.S[cur ^ 1][f] + g); }
    }
    if (P.manning) {
      for (int f = 0; f < 4; ++f)
        if (P.man_p[f]) prefetch_l1(P.man_p[f] + g);
    }
    if (P.irate) { prefetch_l1(P.irate + g); prefetch_l1(P.icap + g); }
    if (P.efx) { prefetch_l1(P.efx + g); prefetch_l1(P.efy + g); }
    if (fc.rain_kind == 3) prefetch_l1(P.pat + g);
    if (fc.rain_kind == 2) { prefetch_l1(P.q0p + g); prefetch_l1(P.q1p + g); }
    if (fc.head_kind == 2) { prefetch_l1(P.hb0p + g); prefetch_l1(P.hb1p + g); }
  };

  for (int k = y0 - 2; k <= y0 + TY + 1; ++k) {
    prefetch_rows(k);
    // row k is loaded where it enters the window: the L1 prefetch issued three iterations
    // earlier has brought it in, and not holding it a row ahead in registers leaves room
    // for more resident warps
    Rm = R0; R0 = Rp; Rp = load_row(k);
    if constexpr (EDDY) { Smm_uy = Sm.uy; Smm_vy = Sm.vy; }
    Sm = S0;
    fyA[0] = fyB[0]; fyA[1] = fyB[1]; fyA[2] = fyB[2];
    // forward y quotients between rows k-1 and k
    if (k >= y0 - 1) {
      fyB[0] = divy(Rp.h - R0.h);
      fyB[1] = divy(Rp.u - R0.u);
      fyB[2] = divy(Rp.v - R0.v);
    }
    // slopes of row k-1 (State.cpp:187-192): Y axis uses north (row k) as the left neighbour
    if (k >= y0) {
      const int r = k - 1;
      const bool hasN = r < ny - 1, hasS = r > 0;
      S0.hy = minmod3q<T>(-fyB[0], hasN, -fyA[0], hasS, divy(Rm.h - Rp.h));
      S0.uy = minmod3q<T>(-fyB[1], hasN, -fyA[1], hasS, divy(Rm.u - Rp.u));
      S0.vy = minmod3q<T>(-fyB[2], hasN, -fyA[2], hasS, divy(Rm.v - Rp.v));
      {
        T r_ = dn1(R0.h), l_ = up1(R0.h);
        T fq = divx(r_ - R0.h);
        S0.hx = minmod3q<T>(up1(fq), hasW, fq, hasE, divx(r_ - l_));
      }
      {
        T r_ = dn1(R0.u), l_ = up1(R0.u);
        T fq = divx(r_ - R0.u);
        S0.ux = minmod3q<T>(up1(fq), hasW, fq, hasE, divx(r_ - l_));
      }
      {
        T r_ = dn1(R0.v), l_ = up1(R0.v);
        T fq = divx(r_ - R0.v);
        S0.vx = minmod3q<T>(up1(fq), hasW, fq, hasE, divx(r_ - l_));
      }
    }
    // horizontal face between rows k-2 and k-1 (face row fy = k-1), Fluxes.cpp:55-64
    if (k >= y0 + 1 && out_lane) {
      const int fy = k - 1;
      if (fy <= ny) {
        const int edge = fy == 0 ? -1 : (fy == ny ? 1 : 0);
        const CellV<T> lo = mkcell(Rm, Sm), hi = mkcell(R0, S0);
        if (P.zdat && edge == 0) {
          CellV<T> lo2 = lo, hi2 = hi;
          face_frame<T>(P, lo2, hi2, gx, fy - 1, gx, fy);
          face_flux<T, 1>(lo2, hi2, edge, hdy, divy, FN);
        } else {
          face_flux<T, 1>(edge == -1 ? hi : lo, edge == 1 ? lo : hi, edge, hdy, divy, FN);
        }
      }
    }
    // output row k-2
    if (k >= y0 + 2) {
      const int r = k - 2;
      const CellV<T> me = mkcell(Rm, Sm);
      const CellV<T> lf = shfl_cell_up(me);
      EddyIn<T> ed{};
      if constexpr (EDDY) {
        if (P.eddy) {  // second derivatives of row r: x by shuffles, y from rows r+1, r, r-1
          ed.ux = Sm.ux; ed.uy = Sm.uy; ed.vx = Sm.vx; ed.vy = Sm.vy;
          {
            T r_ = dn1(Sm.ux), l_ = up1(Sm.ux);
            T fq = divx(r_ - Sm.ux);
            ed.uxx = minmod3q<T>(up1(fq), hasW, fq, hasE, divx(r_ - l_));
          }
          {
            T r_ = dn1(Sm.vx), l_ = up1(Sm.vx);
            T fq = divx(r_ - Sm.vx);
            ed.vxx = minmod3q<T>(up1(fq), hasW, fq, hasE, divx(r_ - l_));
          }
          const bool hasN = r < ny - 1, hasS = r > 0;  // Y axis: north is the left neighbour
          ed.uyy = minmod3q<T>(divy(Sm.uy - S0.uy), hasN, divy(Smm_uy - Sm.uy), hasS, divy(Smm_uy - S0.uy));
          ed.vyy = minmod3q<T>(divy(Sm.vy - S0.vy), hasN, divy(Smm_vy - Sm.vy), hasS, divy(Smm_vy - S0.vy));
        }
      }
      FaceF<T> FW{T(0), T(0), T(0), T(0)};
      if (wface_lane && r < ny) {
        const int edge = gx == 0 ? -1 : (gx == nx ? 1 : 0);
        if (P.zdat && edge == 0) {
          CellV<T> lf2 = lf, me2 = me;
          face_frame<T>(P, lf2, me2, gx - 1, r, gx, r);
          face_flux<T, 0>(lf2, me2, edge, hdx, divx, FW);
        } else {
          face_flux<T, 0>(edge == -1 ? me : lf, edge == 1 ? lf : me, edge, hdx, divx, FW);
        }
      }
      const FaceF<T> FE{dn1(FW.h), dn1(FW.u), dn1(FW.v), dn1(FW.z)};
      if (out_lane && r < ny) {
        const long long g = (long long)r * nx + gx;
        finish_cell<T, CellCtx<T, DX>, EDDY, true, COH>(P, fc, c, g, gx, r, me.h, me.u, me.v, me.dhdx, me.dhdy,
                                                        me.dzdx, me.dzdy, FW, FE, FS, FN, first, last, cur, dt_d, rain,
                                                        removed, walls, xcfl, xmin, vol, &ed);
      }
    }
    FS = FN;
  }
  if (last && !(P.mode & M_DEBUGK)) {
    double mx = warp_max(double(xcfl)), mn = warp_min(double(xmin)), vs = warp_sum<T>(vol);
    if (lane == 0) {
      P.part[gw] = mx;
      P.part[P.nblk + gw] = mn;
      P.part[2 * P.nblk + gw] = vs;
    }
  }
  if (P.mode & M_TALLY) {
    double rs = warp_sum<T>(rain), os = warp_sum<T>(removed), ws = warp_sum<T>(walls);
    if (lane == 0) {
      P.part[(3 + 3LL * P.stage) * P.nblk + gw] = rs;
      P.part[(4 + 3LL * P.stage) * P.nblk + gw] = os;
      P.part[(5 + 3LL * P.stage) * P.nblk + gw] = ws;
    }
  }
}

// Whether strip `gw` of the column sweep with TY output rows is interior: its window (the
// 32 columns x TY + 4 rows of cells it loads) lies inside the mesh with a cell to spare on
// every side. Every slope it computes is then two-sided, none of its faces is a mesh-edge face
// and none of its output cells lies on an edge strip.
__host__ __device__ inline bool strip_inside(long long gw, int nx, int ny, int ty) {
  const int tiles_x = (nx + kSweepOut - 1) / kSweepOut;
  const int x0 = int(gw % tiles_x) * kSweepOut, y0 = int(gw / tiles_x) * ty;
  return x0 >= 2 && x0 + 30 <= nx && y0 >= 2 && y0 + ty + 2 <= ny;
}

// Per strip: 1 for an interior strip whose window holds no coded-out (NaN) bed, so that no
// edge or coded-out mask applies to any of its faces; else 0. One warp per strip.
template <typename T>
__global__ void strip_flags_kernel(const T* __restrict__ z, int nx, int ny, int ty, long long nstrips,
                                   unsigned char* __restrict__ flag) {
  const long long gw = (long long)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  if (gw >= nstrips) return;  // whole warp
  const int lane = threadIdx.x & 31;
  bool ok = strip_inside(gw, nx, ny, ty);
  if (ok) {
    const int tiles_x = (nx + kSweepOut - 1) / kSweepOut;
    const int gx = int(gw % tiles_x) * kSweepOut - 2 + lane, y0 = int(gw / tiles_x) * ty;
    for (int r = y0 - 2; r <= y0 + ty + 1; ++r) {
      const T v = z[(long long)r * nx + gx];
      if (v != v) ok = false;
    }
  }
  ok = __all_sync(kFull, ok);
  if (lane == 0) flag[gw] = ok ? 1 : 0;
}

// One interior strip (strip_flags_kernel) of one solver's stage: the column sweep of
// sweep_strip with every neighbour present and no mask to apply. The face fluxes are formed
// from reconstructed face sides (side_m / side_p, then face_combine): each lane reconstructs
// its east side once and its east neighbour takes those four values by shuffles. In FP64 the
// arithmetic is the general path's, operation for operation; in FP32 the tangential
// finiteness tests are dropped (they only matter for slopes that are not finite, which an
// interior window without coded-out beds produces only from a non-finite state).
template <typename T, int TY, bool P2, bool EDDY, bool COH = false>
__device__ __forceinline__ void sweep_strip_interior(const StageParams<T>& P, long long gw) {
  using DX = DivX<T, P2>;
  constexpr bool TCHK = sizeof(T) == 8;
  const Ctl* ctl = P.ctl;
  const int nx = P.nx, ny = P.ny;
  const int tiles_x = (nx + kSweepOut - 1) / kSweepOut;
  const int lane = threadIdx.x;
  const int tile_x = int(gw % tiles_x), tile_y = int(gw / tiles_x);
  const int gx = tile_x * kSweepOut - 2 + lane;  // inside the mesh for every lane
  const bool out_lane = lane >= 2 && lane < 2 + kSweepOut;
  const int y0 = tile_y * TY;

  const int cur = ctl->cur;
  const double dt_d = ctl->dt;
  const double tsub = ctl->t_local + P.c_s * dt_d;
  const bool first = P.mode & M_FIRST, last = P.mode & M_LAST;
  const T* Yh = first ? P.S[cur][0] : P.Yin[0];
  const T* Yu = first ? P.S[cur][1] : P.Yin[1];
  const T* Yv = first ? P.S[cur][2] : P.Yin[2];
  const DX divx = MkDivX<DX>::make(P.dx), divy = MkDivX<DX>::make(P.dy);
  const T hdx = T(0.5) * T(P.dx), hdy = T(0.5) * T(P.dy);
  CellCtx<T, DX> c;
  c.divx = divx; c.divy = divy;
  c.divdt = mkdiv<T>(dt_d);
  c.divL = mkdiv<T>(P.L);
  c.dt = T(dt_d); c.dt_d = dt_d; c.tsub_d = tsub;
  c.manning = P.manning; c.rain_mode = P.rain_mode; c.head_first = P.head_first;
  const DevForcing fc = *P.fc;
  // FP32 with tile datums: a vertical face crosses datum tiles where its right cell starts a
  // tile column, a horizontal face where its upper row starts a tile row; there the upper /
  // right cell's bed moves into the other cell's frame (face_frame)
  const bool xcross = P.zdat != nullptr && (gx % kDatumTX) == 0;

  auto load_row = [&](int r) {
    const long long g = (long long)r * nx + gx;
    RowV<T> v;
    v.h = ldst<COH>(Yh, g); v.u = ldst<COH>(Yu, g); v.v = ldst<COH>(Yv, g);
    v.z = ld(P.z, g);
    v.zx = ld(P.zx, g); v.zy = ld(P.zy, g);
    return v;
  };
  PfPlan<T> pf;
  pf.init(P, fc, Yh, Yu, Yv, first, cur, gx - lane, lane);

  RowV<T> Rm{}, R0{}, Rp{};
  SlopeV<T> Sm{}, S0{};
  T Smm_uy = T(0), Smm_vy = T(0);
  T fyA[3] = {}, fyB[3] = {};
  FaceF<T> FS{}, FN{};
  double rain = 0.0, removed = 0.0, walls = 0.0, vol = 0.0;
  T xcfl = T(0), xmin = T(1.0 / 0.0);
  T xstep = T(0);  // datum step of the west face in the current tile row (xcross lanes)

  for (int k = y0 - 2; k <= y0 + TY + 1; ++k) {
    pf.rows(k, nx, ny);
    Rm = R0; R0 = Rp; Rp = load_row(k);
    if constexpr (EDDY) { Smm_uy = Sm.uy; Smm_vy = Sm.vy; }
    Sm = S0;
    fyA[0] = fyB[0]; fyA[1] = fyB[1]; fyA[2] = fyB[2];
    if (k >= y0 - 1) {
      fyB[0] = divy(Rp.h - R0.h);
      fyB[1] = divy(Rp.u - R0.u);
      fyB[2] = divy(Rp.v - R0.v);
    }
    // slopes of row k-1 (State.cpp:187-192), two-sided; the Y axis uses north as the left side
    if (k >= y0) {
      S0.hy = slope2s<T>(-fyB[0], -fyA[0], divy(Rm.h - Rp.h));
      S0.uy = slope2s<T>(-fyB[1], -fyA[1], divy(Rm.u - Rp.u));
      S0.vy = slope2s<T>(-fyB[2], -fyA[2], divy(Rm.v - Rp.v));
      {
        T r_ = dn1(R0.h), l_ = up1(R0.h);
        T fq = divx(r_ - R0.h);
        S0.hx = slope2s<T>(up1(fq), fq, divx(r_ - l_));
      }
      {
        T r_ = dn1(R0.u), l_ = up1(R0.u);
        T fq = divx(r_ - R0.u);
        S0.ux = slope2s<T>(up1(fq), fq, divx(r_ - l_));
      }
      {
        T r_ = dn1(R0.v), l_ = up1(R0.v);
        T fq = divx(r_ - R0.v);
        S0.vx = slope2s<T>(up1(fq), fq, divx(r_ - l_));
      }
    }
    // horizontal face between rows k-2 and k-1 (face row fy = k-1), Fluxes.cpp:55-64
    if (k >= y0 + 1 && out_lane) {
      const int fy = k - 1;
      const CellV<T> lo = mkcell(Rm, Sm);
      CellV<T> hi = mkcell(R0, S0);
      if (P.zdat != nullptr && (fy % kDatumTY) == 0) {
        const long long tb = datum_tile(gx, fy, P.dtiles_x);
        hi.z = T(double(hi.z) + (P.zdat[tb] - P.zdat[tb - P.dtiles_x]));
      }
      face_combine<T, 1, TCHK>(side_m<T, 1, TCHK>(lo, hdy), side_p<T, 1, TCHK>(hi, hdy), divy, FN);
    }
    // output row k-2
    if (k >= y0 + 2) {
      const int r = k - 2;
      const CellV<T> me = mkcell(Rm, Sm);
      EddyIn<T> ed{};
      if constexpr (EDDY) {
        if (P.eddy) {  // second derivatives of row r: x by shuffles, y from rows r+1, r, r-1
          ed.ux = Sm.ux; ed.uy = Sm.uy; ed.vx = Sm.vx; ed.vy = Sm.vy;
          {
            T r_ = dn1(Sm.ux), l_ = up1(Sm.ux);
            T fq = divx(r_ - Sm.ux);
            ed.uxx = slope2s<T>(up1(fq), fq, divx(r_ - l_));
          }
          {
            T r_ = dn1(Sm.vx), l_ = up1(Sm.vx);
            T fq = divx(r_ - Sm.vx);
            ed.vxx = slope2s<T>(up1(fq), fq, divx(r_ - l_));
          }
          ed.uyy = slope2s<T>(divy(Sm.uy - S0.uy), divy(Smm_uy - Sm.uy), divy(Smm_uy - S0.uy));
          ed.vyy = slope2s<T>(divy(Sm.vy - S0.vy), divy(Smm_vy - Sm.vy), divy(Smm_vy - S0.vy));
        }
      }
      // west face: the left lane's east side against this lane's west side
      const Side<T> mE = side_m<T, 0, TCHK>(me, hdx);
      const Side<T> mW{up1(mE.zb), up1(mE.h), up1(mE.un), up1(mE.ut)};
      CellV<T> meW = me;
      if (xcross) {
        // the datum step across the tile column edge, read once per tile row: datums are
        // multiples of 2^-10 m, so the step is exact in FP32 (below 2^14 m) and me.z + step
        // rounds as the FP64 sum does; an inexact step (NaN here) takes the FP64 sum
        if (r == y0 || (r % kDatumTY) == 0) {
          const long long tb = datum_tile(gx, r, P.dtiles_x);
          const double st = P.zdat[tb] - P.zdat[tb - 1];
          xstep = double(T(st)) == st ? T(st) : Lim<T>::nan();
        }
        if (xstep == xstep) {
          meW.z = me.z + xstep;
        } else {
          const long long tb = datum_tile(gx, r, P.dtiles_x);
          meW.z = T(double(me.z) + (P.zdat[tb] - P.zdat[tb - 1]));
        }
      }
      FaceF<T> FW;
      face_combine<T, 0, TCHK>(mW, side_p<T, 0, TCHK>(meW, hdx), divx, FW);
      const FaceF<T> FE{dn1(FW.h), dn1(FW.u), dn1(FW.v), dn1(FW.z)};
      if (out_lane) {
        const long long g = (long long)r * nx + gx;
        finish_cell<T, CellCtx<T, DX>, EDDY, false, COH>(P, fc, c, g, gx, r, me.h, me.u, me.v, me.dhdx, me.dhdy,
                                                    me.dzdx, me.dzdy, FW, FE, FS, FN, first, last, cur, dt_d, rain,
                                                    removed, walls, xcfl, xmin, vol, &ed);
      }
    }
    FS = FN;
  }
  if (last && !(P.mode & M_DEBUGK)) {
    double mx = warp_max(double(xcfl)), mn = warp_min(double(xmin)), vs = warp_sum<T>(vol);
    if (lane == 0) {
      P.part[gw] = mx;
      P.part[P.nblk + gw] = mn;
      P.part[2 * P.nblk + gw] = vs;
    }
  }
  if (P.mode & M_TALLY) {
    double rs = warp_sum<T>(rain), os = warp_sum<T>(removed), ws = warp_sum<T>(walls);
    if (lane == 0) {
      P.part[(3 + 3LL * P.stage) * P.nblk + gw] = rs;
      P.part[(4 + 3LL * P.stage) * P.nblk + gw] = os;
      P.part[(5 + 3LL * P.stage) * P.nblk + gw] = ws;
    }
  }
}

// The column sweeps of one stage are split over disjoint strip lists (general, interior,
// interior pairs) that read the same inputs and write disjoint cells and partial slots. Each
// of them lets the launch queued after it start at once (programmatic dependent launch: the
// launcher marks the next sweep of the same stage as allowed to overlap), so the small
// general launch over the edge strips runs beside the interior ones instead of as a tail. A
// launch not marked that way (the next stage, the finalize) still waits for all of them.
__device__ __forceinline__ void allow_overlap() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// The general column sweep over the strips in P.bstrips (every strip when the list is null).
template <typename T, int TY, int WPB, int MINB, bool P2, bool EDDY>
__global__ void __launch_bounds__(32 * WPB, MINB) sweep_kernel(const __grid_constant__ StageParams<T> P) {
  allow_overlap();
  if (P.ctl->done) return;
  const long long i = (long long)blockIdx.x * WPB + threadIdx.y;
  long long gw = i;
  if (P.bstrips) {
    if (i >= P.n_bstrips) return;  // whole warp: no block-level synchronisation below
    gw = P.bstrips[i];
  } else {
    const int tiles_x = (P.nx + kSweepOut - 1) / kSweepOut;
    if (i >= (long long)tiles_x * ((P.ny + TY - 1) / TY)) return;
  }
  sweep_strip<T, TY, P2, EDDY>(P, gw);
}

// The interior column sweep over the strips in P.istrips.
template <typename T, int TY, int WPB, int MINB, bool P2, bool EDDY>
__global__ void __launch_bounds__(32 * WPB, MINB) sweep_interior_kernel(const __grid_constant__ StageParams<T> P) {
  allow_overlap();
  if (P.ctl->done) return;
  const long long i = (long long)blockIdx.x * WPB + threadIdx.y;
  if (i >= P.n_istrips) return;  // whole warp
  sweep_strip_interior<T, TY, P2, EDDY>(P, P.istrips[i]);
}

// ---------------------------------------------------------------------------------------
// Interior column sweep with two cells per lane (FP32). One warp sweeps a pair of adjacent
// interior strips, 2 x kSweepOut = 56 output columns: lane l holds columns gx0 + 2l and
// gx0 + 2l + 1 (gx0 = the pair's first output column - 2) and loads both as one 8-byte
// vector per field. Lanes 1-28 write output; lanes 0 and 29 hold the two-column halo; lanes
// 30-31 hold nothing that is used (their loads are clamped into the mesh). Per pair of cells
// the x neighbours take three shuffles per field (the left lane's second cell, the right
// lane's first cell and the left lane's right difference quotient) and the vertical faces
// eight (the left lane's east face side, the right lane's west face flux), half of what the
// one-cell sweep needs; the face between a lane's two cells needs none. The arithmetic per
// face and per cell is the interior sweep's.
// ---------------------------------------------------------------------------------------
template <int TY, bool P2, bool EDDY>
__device__ __forceinline__ void sweep_pair_interior(const StageParams<float>& P, long long gw) {
  using T = float;
  using DX = DivX<T, P2>;
  const Ctl* ctl = P.ctl;
  const int nx = P.nx, ny = P.ny;
  const int tiles_x = (nx + kSweepOut - 1) / kSweepOut;
  const int lane = threadIdx.x;
  const int tile_x = int(gw % tiles_x), tile_y = int(gw / tiles_x);  // the pair's first strip
  const int ca = tile_x * kSweepOut - 2 + 2 * lane;                    // columns ca, ca + 1
  const int lc = min(ca, nx - 2);  // load column: even (nx is even for pairs), inside the mesh
  const bool out_lane = lane >= 1 && lane <= kSweepOut;
  const int y0 = tile_y * TY;

  const int cur = ctl->cur;
  const double dt_d = ctl->dt;
  const double tsub = ctl->t_local + P.c_s * dt_d;
  const bool first = P.mode & M_FIRST, last = P.mode & M_LAST;
  const T* Yh = first ? P.S[cur][0] : P.Yin[0];
  const T* Yu = first ? P.S[cur][1] : P.Yin[1];
  const T* Yv = first ? P.S[cur][2] : P.Yin[2];
  const DX divx = MkDivX<DX>::make(P.dx), divy = MkDivX<DX>::make(P.dy);
  const T hdx = T(0.5) * T(P.dx), hdy = T(0.5) * T(P.dy);
  CellCtx<T, DX> c;
  c.divx = divx; c.divy = divy;
  c.divdt = mkdiv<T>(dt_d);
  c.divL = mkdiv<T>(P.L);
  c.dt = T(dt_d); c.dt_d = dt_d; c.tsub_d = tsub;
  c.manning = P.manning; c.rain_mode = P.rain_mode; c.head_first = P.head_first;
  const DevForcing fc = *P.fc;
  // tile datums: the first cell of a lane can start a datum tile column (the second one, at an
  // odd column, never does), so only the west face of the first cell crosses tiles in x
  const bool xcross = P.zdat != nullptr && (ca % kDatumTX) == 0;

  auto ld2 = [&](const T* p, long long g) { return __ldg(reinterpret_cast<const float2*>(p + g)); };
  auto load_row = [&](int r, RowV<T>& A, RowV<T>& B) {
    const long long g = (long long)r * nx + lc;
    float2 t;
    t = ld2(Yh, g); A.h = t.x; B.h = t.y;
    t = ld2(Yu, g); A.u = t.x; B.u = t.y;
    t = ld2(Yv, g); A.v = t.x; B.v = t.y;
    t = ld2(P.z, g); A.z = t.x; B.z = t.y;
    t = ld2(P.zx, g); A.zx = t.x; B.zx = t.y;
    t = ld2(P.zy, g); A.zy = t.x; B.zy = t.y;
  };
  auto prefetch_rows = [&](int k) {
    {
      const int r = min(k + 1 + kSweepPfWindow, ny - 1);
      const long long g = (long long)r * nx + lc;
      prefetch_l1(Yh + g); prefetch_l1(Yu + g); prefetch_l1(Yv + g);
      prefetch_l1(P.z + g); prefetch_l1(P.zx + g); prefetch_l1(P.zy + g);
    }
    const int r = min(k - 2 + kSweepPfCell, ny - 1);
    const long long g = (long long)r * nx + lc;
    if (!first) {
      for (int f = 0; f < 3; ++f) { prefetch_l1(P.S[cur][f] + g); prefetch_l1(P.S[cur ^ 1][f] + g); }
    }
    if (P.manning) {
      for (int f = 0; f < 4; ++f)
        if (P.man_p[f]) prefetch_l1(P.man_p[f] + g);
    }
    if (P.irate) { prefetch_l1(P.irate + g); prefetch_l1(P.icap + g); }
    if (P.efx) { prefetch_l1(P.efx + g); prefetch_l1(P.efy + g); }
    if (fc.rain_kind == 3) prefetch_l1(P.pat + g);
    if (fc.rain_kind == 2) { prefetch_l1(P.q0p + g); prefetch_l1(P.q1p + g); }
    if (fc.head_kind == 2) { prefetch_l1(P.hb0p + g); prefetch_l1(P.hb1p + g); }
  };
  // x slopes of a lane's two cells (values A, B) from their neighbours in the adjacent lanes
  auto xslopes = [&](T A, T B, T& sa, T& sb) {
    const T Bl = up1(B);          // column ca - 1
    const T Ar = dn1(A);          // column ca + 2
    const T qab = divx(B - A);
    const T qbr = divx(Ar - B);
    const T qla = up1(qbr);       // (A - Bl) / dx, formed by the left lane
    sa = minmod3_finite(qla, qab, divx(B - Bl));
    sb = minmod3_finite(qab, qbr, divx(Ar - A));
  };

  RowV<T> Rm[2] = {}, R0[2] = {}, Rp[2] = {};
  SlopeV<T> Sm[2] = {}, S0[2] = {};
  T Smm_uy[2] = {}, Smm_vy[2] = {};
  T fyA[2][3] = {}, fyB[2][3] = {};
  FaceF<T> FS[2] = {}, FN[2] = {};
  double rain = 0.0, removed = 0.0, walls = 0.0, vol = 0.0;
  T xcfl = T(0), xmin = T(1.0 / 0.0);

  for (int k = y0 - 2; k <= y0 + TY + 1; ++k) {
    prefetch_rows(k);
#pragma unroll
    for (int j = 0; j < 2; ++j) { Rm[j] = R0[j]; R0[j] = Rp[j]; }
    load_row(k, Rp[0], Rp[1]);
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      if constexpr (EDDY) { Smm_uy[j] = Sm[j].uy; Smm_vy[j] = Sm[j].vy; }
      Sm[j] = S0[j];
      fyA[j][0] = fyB[j][0]; fyA[j][1] = fyB[j][1]; fyA[j][2] = fyB[j][2];
      if (k >= y0 - 1) {
        fyB[j][0] = divy(Rp[j].h - R0[j].h);
        fyB[j][1] = divy(Rp[j].u - R0[j].u);
        fyB[j][2] = divy(Rp[j].v - R0[j].v);
      }
    }
    // slopes of row k-1 (State.cpp:187-192), two-sided; the Y axis uses north as the left side
    if (k >= y0) {
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        S0[j].hy = minmod3_finite(-fyB[j][0], -fyA[j][0], divy(Rm[j].h - Rp[j].h));
        S0[j].uy = minmod3_finite(-fyB[j][1], -fyA[j][1], divy(Rm[j].u - Rp[j].u));
        S0[j].vy = minmod3_finite(-fyB[j][2], -fyA[j][2], divy(Rm[j].v - Rp[j].v));
      }
      xslopes(R0[0].h, R0[1].h, S0[0].hx, S0[1].hx);
      xslopes(R0[0].u, R0[1].u, S0[0].ux, S0[1].ux);
      xslopes(R0[0].v, R0[1].v, S0[0].vx, S0[1].vx);
    }
    // horizontal faces between rows k-2 and k-1 (face row fy = k-1), Fluxes.cpp:55-64
    if (k >= y0 + 1 && out_lane) {
      const int fy = k - 1;
      double dz = 0.0;
      const bool ycross = P.zdat != nullptr && (fy % kDatumTY) == 0;
      if (ycross) {  // both cells of the lane lie in one datum tile column
        const long long tb = datum_tile(ca, fy, P.dtiles_x);
        dz = P.zdat[tb] - P.zdat[tb - P.dtiles_x];
      }
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const CellV<T> lo = mkcell(Rm[j], Sm[j]);
        CellV<T> hi = mkcell(R0[j], S0[j]);
        if (ycross) hi.z = T(double(hi.z) + dz);
        face_combine<T, 1, false>(side_m<T, 1, false>(lo, hdy), side_p<T, 1, false>(hi, hdy), divy, FN[j]);
      }
    }
    // output row k-2
    if (k >= y0 + 2) {
      const int r = k - 2;
      const CellV<T> meA = mkcell(Rm[0], Sm[0]), meB = mkcell(Rm[1], Sm[1]);
      EddyIn<T> ed[2] = {};
      if constexpr (EDDY) {
        if (P.eddy) {  // second derivatives of row r: x from the lanes' slopes, y from rows r+1, r, r-1
#pragma unroll
          for (int j = 0; j < 2; ++j) {
            ed[j].ux = Sm[j].ux; ed[j].uy = Sm[j].uy; ed[j].vx = Sm[j].vx; ed[j].vy = Sm[j].vy;
            ed[j].uyy = minmod3_finite(divy(Sm[j].uy - S0[j].uy), divy(Smm_uy[j] - Sm[j].uy),
                                       divy(Smm_uy[j] - S0[j].uy));
            ed[j].vyy = minmod3_finite(divy(Sm[j].vy - S0[j].vy), divy(Smm_vy[j] - Sm[j].vy),
                                       divy(Smm_vy[j] - S0[j].vy));
          }
          xslopes(Sm[0].ux, Sm[1].ux, ed[0].uxx, ed[1].uxx);
          xslopes(Sm[0].vx, Sm[1].vx, ed[0].vxx, ed[1].vxx);
        }
      }
      // west face of the first cell: the left lane's second cell's east side against it
      const Side<T> eB = side_m<T, 0, false>(meB, hdx);
      const Side<T> wA{up1(eB.zb), up1(eB.h), up1(eB.un), up1(eB.ut)};
      CellV<T> meAW = meA;
      if (xcross) {
        const long long tb = datum_tile(ca, r, P.dtiles_x);
        meAW.z = T(double(meA.z) + (P.zdat[tb] - P.zdat[tb - 1]));
      }
      FaceF<T> FWa, Fab;
      face_combine<T, 0, false>(wA, side_p<T, 0, false>(meAW, hdx), divx, FWa);
      // the face between the lane's two cells
      face_combine<T, 0, false>(side_m<T, 0, false>(meA, hdx), side_p<T, 0, false>(meB, hdx), divx, Fab);
      // east face of the second cell: the right lane's west face
      const FaceF<T> FEb{dn1(FWa.h), dn1(FWa.u), dn1(FWa.v), dn1(FWa.z)};
      if (out_lane) {
        const long long g = (long long)r * nx + ca;
        finish_cell<T, CellCtx<T, DX>, EDDY, false>(P, fc, c, g, ca, r, meA.h, meA.u, meA.v, meA.dhdx, meA.dhdy,
                                                    meA.dzdx, meA.dzdy, FWa, Fab, FS[0], FN[0], first, last, cur,
                                                    dt_d, rain, removed, walls, xcfl, xmin, vol, &ed[0]);
        finish_cell<T, CellCtx<T, DX>, EDDY, false>(P, fc, c, g + 1, ca + 1, r, meB.h, meB.u, meB.v, meB.dhdx,
                                                    meB.dhdy, meB.dzdx, meB.dzdy, Fab, FEb, FS[1], FN[1], first, last,
                                                    cur, dt_d, rain, removed, walls, xcfl, xmin, vol, &ed[1]);
      }
    }
    FS[0] = FN[0];
    FS[1] = FN[1];
  }
  // the pair's partials go to its first strip's slot; the second strip's slot gets the
  // identities (max 0, min +inf, sums 0)
  if (last && !(P.mode & M_DEBUGK)) {
    double mx = warp_max(double(xcfl)), mn = warp_min(double(xmin)), vs = warp_sum<T>(vol);
    if (lane == 0) {
      P.part[gw] = mx;
      P.part[P.nblk + gw] = mn;
      P.part[2 * P.nblk + gw] = vs;
      P.part[gw + 1] = 0.0;
      P.part[P.nblk + gw + 1] = 1.0 / 0.0;
      P.part[2 * P.nblk + gw + 1] = 0.0;
    }
  }
  if (P.mode & M_TALLY) {
    double rs = warp_sum<T>(rain), os = warp_sum<T>(removed), ws = warp_sum<T>(walls);
    if (lane == 0) {
      P.part[(3 + 3LL * P.stage) * P.nblk + gw] = rs;
      P.part[(4 + 3LL * P.stage) * P.nblk + gw] = os;
      P.part[(5 + 3LL * P.stage) * P.nblk + gw] = ws;
      P.part[(3 + 3LL * P.stage) * P.nblk + gw + 1] = 0.0;
      P.part[(4 + 3LL * P.stage) * P.nblk + gw + 1] = 0.0;
      P.part[(5 + 3LL * P.stage) * P.nblk + gw + 1] = 0.0;
    }
  }
}

// The two-cells-per-lane interior sweep over the strip pairs in P.ipairs (each entry the
// pair's first strip).
template <int TY, int WPB, int MINB, bool P2, bool EDDY>
__global__ void __launch_bounds__(32 * WPB, MINB) sweep_pair_kernel(const __grid_constant__ StageParams<float> P) {
  allow_overlap();
  if (P.ctl->done) return;
  const long long i = (long long)blockIdx.x * WPB + threadIdx.y;
  if (i >= P.n_ipairs) return;  // whole warp
  sweep_pair_interior<TY, P2, EDDY>(P, P.ipairs[i]);
}

// Batched column sweep: the strips of every instance of a batch, warp_start[i] being the
// first global warp of instance i. Each warp finds its instance, stages its parameters in
// shared memory and sweeps its strip; instances whose step is finished return at once.
template <typename T, int TY, int WPB, int MINB, bool P2, bool EDDY>
__global__ void __launch_bounds__(32 * WPB, MINB)
    sweep_batch_kernel(const StageParams<T>* __restrict__ Ps, const long long* __restrict__ warp_start, int ninst) {
  __shared__ __align__(16) StageParams<T> Psh[WPB];
  const long long gw = (long long)blockIdx.x * WPB + threadIdx.y;
  if (gw >= warp_start[ninst]) return;  // whole warp
  int inst = 0;
  if (threadIdx.x == 0) {
    int lo = 0, hi = ninst - 1;  // last instance with warp_start[i] <= gw
    while (lo < hi) {
      int mid = (lo + hi + 1) / 2;
      if (warp_start[mid] <= gw) lo = mid;
      else hi = mid - 1;
    }
    inst = lo;
  }
  inst = __shfl_sync(kFull, inst, 0);
  static_assert(sizeof(StageParams<T>) % 4 == 0, "parameter block copied as 32-bit words");
  const unsigned* src = reinterpret_cast<const unsigned*>(Ps + inst);
  unsigned* dst = reinterpret_cast<unsigned*>(&Psh[threadIdx.y]);
  for (int i = threadIdx.x; i < int(sizeof(StageParams<T>) / 4); i += 32) dst[i] = src[i];
  __syncwarp();
  const StageParams<T>& P = Psh[threadIdx.y];
  if (P.ctl->done) return;
  sweep_strip<T, TY, P2, EDDY>(P, gw - warp_start[inst]);
}

// Bed slopes once per bed upload (SaintVenantConstants, Constants.cpp:39-40).
// The slopes are computed in T and stored as TO (FP32 with tile datums: FP64 slopes of the
// FP64 bed, rounded once).
template <typename T, typename TO = T>
__global__ void bed_slopes_kernel(const T* z, int nx, int ny, double dx, double dy, TO* zx, TO* zy) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long n = (long long)nx * ny;
  if (i >= n) return;
  int gx = int(i % nx), gy = int(i / nx);
  bool hasW = gx > 0, hasE = gx < nx - 1, hasN = gy < ny - 1, hasS = gy > 0;
  T cz = z[i];
  zx[i] = TO(minmod3<T>(hasW ? z[i - 1] : cz, hasW, cz, hasE, hasE ? z[i + 1] : cz, mkdiv<T>(dx)));
  zy[i] = TO(minmod3<T>(hasN ? z[i + nx] : cz, hasN, cz, hasS, hasS ? z[i - nx] : cz, mkdiv<T>(dy)));
}

// Fields arrive and leave in FP64 (the interface's type); a solver of another value type
// converts them here, one rounding per value as a host cast would do.
template <typename TI, typename TO>
__global__ void convert_kernel(const TI* __restrict__ src, TO* __restrict__ dst, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[i] = TO(src[i]);
}

// Whether an FP64 field, once converted to T, differs bit for bit from a stored one: sets *flag.
__device__ __forceinline__ bool same_bits(double a, double b) { return __double_as_longlong(a) == __double_as_longlong(b); }
__device__ __forceinline__ bool same_bits(float a, float b) { return __float_as_uint(a) == __float_as_uint(b); }
template <typename T>
__global__ void differs_kernel(const double* __restrict__ src, const T* __restrict__ ref, long long n, int* flag) {
  bool diff = false;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    diff = diff || !same_bits(T(src[i]), ref[i]);
  if (diff) *flag = 1;
}

#ifdef SV_DEFINE_COMMON_KERNELS  // non-template kernels: defined in one unit only
// Datum of each 32 x 8 tile of an FP64 bed: the tile's lowest non-NaN value (among values
// that compare equal, such as -0.0 and 0.0, the first in row-major order), rounded down to a
// multiple of 2^-10 m; 0 for a tile without a valid bed. One warp per tile, a lane per column.
__global__ void datum_tiles_kernel(const double* z, int nx, int ny, int dtiles_x, int dtiles_y, double* zdat) {
  const long long t = (long long)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  if (t >= (long long)dtiles_x * dtiles_y) return;  // whole warp
  const int lane = threadIdx.x & 31;
  const int gx = int(t % dtiles_x) * kDatumTX + lane, ty = int(t / dtiles_x);
  double best = 0.0;
  long long bi = -1;  // row-major index of `best`; -1 = none yet
  if (gx < nx) {
    for (int r = 0; r < kDatumTY; ++r) {
      const int gy = ty * kDatumTY + r;
      if (gy >= ny) break;
      const long long i = (long long)gy * nx + gx;
      const double v = z[i];
      if (v != v) continue;
      if (bi < 0 || v < best) { best = v; bi = i; }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double ob = __shfl_down_sync(kFull, best, o);
    const long long oi = __shfl_down_sync(kFull, bi, o);
    if (oi >= 0 && (bi < 0 || ob < best || (ob == best && oi < bi))) { best = ob; bi = oi; }
  }
  if (lane == 0) zdat[t] = floor((bi < 0 ? 0.0 : best) * 1024.0) / 1024.0;
}

// FP32 offset of each cell's bed from its tile's datum (FP64 difference, rounded once), or the
// absolute FP64 bed from an offset (`to_abs`).
__global__ void datum_offsets_kernel(const double* z, int nx, int ny, int dtiles_x, const double* zdat, float* off) {
  const long long n = (long long)nx * ny;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    off[i] = float(z[i] - zdat[datum_tile(int(i % nx), int(i / nx), dtiles_x)]);
}
__global__ void datum_absolute_kernel(const float* off, int nx, int ny, int dtiles_x, const double* zdat, double* z) {
  const long long n = (long long)nx * ny;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    z[i] = double(off[i]) + zdat[datum_tile(int(i % nx), int(i / nx), dtiles_x)];
}
#endif

// Steps queued for one batch member by one batched advance. The member runs them back to
// back at its own pace: when a step ends, the controller records it and starts the next one
// on the device (TypedTemporalScheme::solve's loop, TemporalScheme.hpp:244-276, moved onto
// the GPU), so members with large timesteps do not wait for the slowest one at every step.
constexpr int kMaxQueuedSteps = 16;
struct StepQueue {
  int n;           // steps queued (0: the member sits this advance out)
  int k;           // steps completed so far
  int status;      // 0, or -5 (time became NaN) / -7 (step limit reached) in step k
  int keep_first;  // 1: step 0 uses the forcing already in place (f[0] unused)
  int cur;         // the member's state parity when the advance ended (host mirror)
  int pad;
  long long limit; // timesteps allowed per step (0: no limit)
  DevForcing f[kMaxQueuedSteps];                             // forcing of each queued step
  unsigned long long acc[kMaxQueuedSteps], rep[kMaxQueuedSteps];   // per-step counts
  double rain[kMaxQueuedSteps], outflow[kMaxQueuedSteps], volume[kMaxQueuedSteps];  // running, at step end
  double wall[kMaxQueuedSteps];
};

struct FinalizeParams {
  Ctl* ctl;
  StepQueue* q;      // batch members: the step queue (null for a solver on its own)
  DevForcing* fc;    // batch members: the member's forcing slot read by its stage kernels
  const double* part;
  long long nblk;
  int nstages;
  double b[4];
  double cn_target, max_dt, L;
  double cell_area;
  int auto_mode;   // 1: accept/repeat, advance t_local, trim dt (TemporalScheme.hpp:119-146)
  int tally;
  int is_float;    // control number rounded to T = float
};

// Fixed-order sum: thread t adds blocks t, t+NT, ... in order, then a fixed tree.
template <int NT> __device__ double fixed_sum(const double* p, long long n, double* red) {
  double a = 0.0;
  for (long long i = threadIdx.x; i < n; i += NT) a += p[i];
  red[threadIdx.x] = a;
  __syncthreads();
  for (int st = NT / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
    __syncthreads();
  }
  double r = red[0];
  __syncthreads();
  return r;
}

__device__ __forceinline__ void finalize_control(const FinalizeParams& F, double mx, double mn, double vol,
                                                 double rain, double outf, double wall);

template <int NT> __device__ __forceinline__ void finalize_body(const FinalizeParams& F, double* red) {
  Ctl* ctl = F.ctl;
  if (ctl->done) return;
  // CFL max / min (NaN-propagating), order-independent
  double mx = 0.0, mn = 1.0 / 0.0;
  for (long long i = threadIdx.x; i < F.nblk; i += NT) {
    mx = nmax(mx, F.part[i]);
    mn = nmin(mn, F.part[F.nblk + i]);
  }
  red[threadIdx.x] = mx;
  __syncthreads();
  for (int st = NT / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) red[threadIdx.x] = nmax(red[threadIdx.x], red[threadIdx.x + st]);
    __syncthreads();
  }
  mx = red[0];
  __syncthreads();
  red[threadIdx.x] = mn;
  __syncthreads();
  for (int st = NT / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) red[threadIdx.x] = nmin(red[threadIdx.x], red[threadIdx.x + st]);
    __syncthreads();
  }
  mn = red[0];
  __syncthreads();
  double vol = fixed_sum<NT>(F.part + 2 * F.nblk, F.nblk, red);
  double rain = 0.0, outf = 0.0, wall = 0.0;
  if (F.tally) {
    for (int s = 0; s < F.nstages; ++s) {
      double rs = fixed_sum<NT>(F.part + (3 + 3LL * s) * F.nblk, F.nblk, red);
      double os = fixed_sum<NT>(F.part + (4 + 3LL * s) * F.nblk, F.nblk, red);
      double ws = fixed_sum<NT>(F.part + (5 + 3LL * s) * F.nblk, F.nblk, red);
      double w = F.is_float ? double(float(F.b[s] * ctl->dt)) : F.b[s] * ctl->dt;
      rain += w * rs * F.cell_area;
      outf += w * os * F.cell_area;
      wall += w * ws * F.cell_area;
    }
  }
  if (threadIdx.x != 0) return;
  finalize_control(F, mx, mn, vol, rain, outf, wall);
}

// The rest of a timestep's finalize, one thread, from its reductions (CFL max and min over
// cells of (|u|+c)/dx + (|v|+c)/dy, volume, tallies): the control number, accept / repeat and
// the new dt (RungeKutta.cpp:154-167), the step clock and the end-of-step trimming
// (TemporalScheme.hpp:119-146) and, for a batch member, its step queue.
__device__ __forceinline__ void finalize_control(const FinalizeParams& F, double mx, double mn, double vol,
                                                 double rain, double outf, double wall) {
  Ctl* ctl = F.ctl;
  const double dt = ctl->dt;
  // control number: max over cells of dt * x
  double cn;
  if (mx != mx || dt != dt) cn = mx + dt;                  // NaN
  else if (dt == 1.0 / 0.0) cn = (mn == 0.0) ? (0.0 / 0.0) : dt;
  else cn = dt * mx;
  if (F.is_float) cn = double(float(cn));
  // RungeKuttaTemporalScheme::do_timestep (RungeKutta.cpp:154-167), target as parameter
  const double tgt = F.cn_target;
  double nd;
  int rep;
  if (cn > tgt) {
    rep = 1;
    nd = (cn > 5.0 * tgt) ? dt / 5.0 : (dt * tgt) / (cn * 1.1);
  } else if (cn > 0.9 * tgt) {
    rep = 0; nd = dt;
  } else {
    rep = 0; nd = (dt * tgt) / cn;
  }
  if (F.max_dt > 0.0 && nd > F.max_dt) nd = F.max_dt;
  ctl->cn = cn;
  ctl->new_dt = nd;
  ctl->repeat = rep;
  ctl->pend_rain = rain;
  ctl->pend_out = outf;
  ctl->pend_wall = wall;
  ctl->pend_vol = vol;
  if (!F.auto_mode) return;
  // TypedTemporalScheme::step (TemporalScheme.hpp:119-146)
  double t = ctl->t_local;
  if (rep) {
    ctl->repeated++; ctl->step_repeated++;
  } else {
    ctl->accepted++; ctl->step_accepted++;
    ctl->rain_in += rain; ctl->outflow += outf; ctl->wall_in += wall; ctl->volume = vol;
    t = t + dt;
    ctl->cur ^= 1;
  }
  double ndt = nd;
  const double L = F.L;
  if (t >= L) {
    ctl->done = 1;
  } else if (t + ndt > L) {
    ndt = L - t;
  } else if (t + 2.0 * ndt > L) {
    ndt = (L - t) * 0.4;
  }
  if (!(t < L) && !(t >= L)) { ctl->done = 1; ctl->error = -5; }   // t became NaN
  ctl->t_local = t;
  ctl->dt = ndt;
  if (ctl->budget > 0 && --ctl->budget == 0 && !ctl->done) ctl->done = 2;  // paused, step not over
  if (F.q == nullptr || !ctl->done) return;
  // batch member: record the step that ended (or failed); start the next queued one
  StepQueue* q = F.q;
  const int k = q->k;
  q->acc[k] = ctl->step_accepted;
  q->rep[k] = ctl->step_repeated;
  q->rain[k] = ctl->rain_in;
  q->outflow[k] = ctl->outflow;
  q->wall[k] = ctl->wall_in;
  q->volume[k] = ctl->volume;
  q->cur = ctl->cur;
  if (ctl->error) { q->status = -5; return; }
  if (ctl->done == 2) { q->status = -7; return; }
  q->k = k + 1;
  if (k + 1 < q->n) {  // start_new_step of the next queued step; dt carries over as in step()
    *F.fc = q->f[k + 1];
    ctl->t_local = 0.0;
    ctl->step_accepted = 0;
    ctl->step_repeated = 0;
    ctl->budget = q->limit;
    ctl->done = 0;
  }
}

template <int NT> __global__ void __launch_bounds__(NT) finalize_kernel(const FinalizeParams F) {
  __shared__ double red[NT];
  finalize_body<NT>(F, red);
}

// Batched finalize: one CTA per instance of a batch.
template <int NT> __global__ void __launch_bounds__(NT) finalize_batch_kernel(const FinalizeParams* __restrict__ Fs) {
  __shared__ double red[NT];
  __shared__ FinalizeParams Fsh;
  if (threadIdx.x == 0) Fsh = Fs[blockIdx.x];
  __syncthreads();
  finalize_body<NT>(Fsh, red);
}

// ---------------------------------------------------------------------------------------
// Persistent batch kernel. One cooperative launch advances every member of a batch through
// its queued steps (TypedTemporalScheme::solve / step for each member, TemporalScheme.hpp:
// 112-149, 244-276), each member at its own dt. A member's timestep is N stage phases of
// column-sweep strips followed by one finalize phase (reductions and the dt controller).
// A warp looks at 32 members at once (one per lane) for one whose open phase has unclaimed
// items and takes that member's next ticket with one atomicAdd (no retry loop, so claims do
// not serialise when many warps work on one member). Tickets number a member's work items in
// order; a ticket past the end of the open phase belongs to a later phase, whose opening its
// warp waits for. The warp that completes the last item of a phase opens the member's next
// phase. Phases are ordered by release fences before each completion count and acquire
// fences before each item, and the state buffers are read with coherent loads (ldst<true>).
// Every wait is bounded twice: a waiting warp gives up after spin_limit polls during which no
// warp completed an item (a global progress count), and every warp gives up once the launch
// has run max_ns; either records SV_E_TIMEOUT in the launch status, and every warp returns at
// its next poll.
// ---------------------------------------------------------------------------------------
struct PersistMember {
  unsigned long long phase;   // phases opened so far: stage = phase % (N + 1), N = the finalize
  unsigned long long ticket;  // work items claimed so far, over all phases
  unsigned int done;          // items of the current phase completed
  int finished;               // 1: no more work for this member in this launch
  long long nstrips;          // column-sweep strips of one stage
};

template <typename T> struct PersistParams {
  const StageParams<T>* Ps;   // stage s of member k at Ps[s * nact + k]
  const FinalizeParams* Fs;   // [nact]
  PersistMember* mem;         // [nact]
  int nact, nstages;
  int* status;                // 0, or SV_E_TIMEOUT (-6) once a wait gave up
  unsigned long long* progress;   // items completed by all warps (zeroed before the launch)
  unsigned long long spin_limit;  // polls without any completed item before giving up
  unsigned long long max_ns;      // wall-clock bound of the launch, ns
};

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

constexpr int kPersistWarps = 4;   // warps per block
constexpr int kPersistRows = 32;   // column-sweep strip height (the batches' variant 8)

#ifdef SV_DEFINE_COMMON_KERNELS
// mark the members whose step queue starts with nothing to do (their controller is done)
__global__ void persist_init_kernel(const FinalizeParams* Fs, PersistMember* mem, const long long* warp_start,
                                    int nact) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nact) return;
  PersistMember m{};
  m.nstrips = warp_start[k + 1] - warp_start[k];
  m.finished = Fs[k].ctl->done != 0 ? 1 : 0;
  mem[k] = m;
}
#endif

// Fixed-order sum of p[0..n) by one warp, in exactly the order of fixed_sum<NT> (thread t of
// NT adds p[t], p[t+NT], ..., then a binary tree): red holds NT doubles.
template <int NT> __device__ double warp_fixed_sum(const double* p, long long n, double* red) {
  const int lane = threadIdx.x & 31;
  for (int t = lane; t < NT; t += 32) {
    double a = 0.0;
    for (long long i = t; i < n; i += NT) a += p[i];
    red[t] = a;
  }
  __syncwarp();
  for (int st = NT / 2; st > 0; st >>= 1) {
    for (int t = lane; t < st; t += 32) red[t] += red[t + st];
    __syncwarp();
  }
  const double r = red[0];
  __syncwarp();
  return r;
}
template <int NT, bool MAX> __device__ double warp_fixed_ext(const double* p, long long n, double* red) {
  const int lane = threadIdx.x & 31;
  for (int t = lane; t < NT; t += 32) {
    double a = MAX ? 0.0 : 1.0 / 0.0;
    for (long long i = t; i < n; i += NT) a = MAX ? nmax(a, p[i]) : nmin(a, p[i]);
    red[t] = a;
  }
  __syncwarp();
  for (int st = NT / 2; st > 0; st >>= 1) {
    for (int t = lane; t < st; t += 32) red[t] = MAX ? nmax(red[t], red[t + st]) : nmin(red[t], red[t + st]);
    __syncwarp();
  }
  const double r = red[0];
  __syncwarp();
  return r;
}

// finalize_body<1024> by one warp: the same reductions in the same order, then the controller
__device__ __forceinline__ void finalize_warp(const FinalizeParams& F, double* red) {
  constexpr int NT = 1024;
  Ctl* ctl = F.ctl;
  const double mx = warp_fixed_ext<NT, true>(F.part, F.nblk, red);
  const double mn = warp_fixed_ext<NT, false>(F.part + F.nblk, F.nblk, red);
  const double vol = warp_fixed_sum<NT>(F.part + 2 * F.nblk, F.nblk, red);
  double rain = 0.0, outf = 0.0, wall = 0.0;
  if (F.tally) {
    for (int s = 0; s < F.nstages; ++s) {
      double rs = warp_fixed_sum<NT>(F.part + (3 + 3LL * s) * F.nblk, F.nblk, red);
      double os = warp_fixed_sum<NT>(F.part + (4 + 3LL * s) * F.nblk, F.nblk, red);
      double ws = warp_fixed_sum<NT>(F.part + (5 + 3LL * s) * F.nblk, F.nblk, red);
      double w = F.is_float ? double(float(F.b[s] * ctl->dt)) : F.b[s] * ctl->dt;
      rain += w * rs * F.cell_area;
      outf += w * os * F.cell_area;
      wall += w * ws * F.cell_area;
    }
  }
  if ((threadIdx.x & 31) == 0) finalize_control(F, mx, mn, vol, rain, outf, wall);
  __syncwarp();
}

template <typename T, bool P2, bool EDDY>
__global__ void __launch_bounds__(32 * kPersistWarps, 4) persist_batch_kernel(const PersistParams<T> PP) {
  __shared__ __align__(16) StageParams<T> Psh[kPersistWarps];
  __shared__ double red[kPersistWarps][1024];
  const int lane = threadIdx.x, wib = threadIdx.y;
  const int N = PP.nstages, nact = PP.nact;
  const long long gwarp = (long long)blockIdx.x * kPersistWarps + wib;
  const int k0 = nact > 0 ? int(gwarp % nact) : 0;
  volatile int* status = PP.status;
  volatile unsigned long long* progress = PP.progress;
  const unsigned long long t_start = global_ns();
  unsigned long long idle = 0, seen = *progress;
  // one poll of a waiting warp; true when the warp must return (another warp gave up, the
  // launch ran out of time, or spin_limit polls passed with no item completed anywhere)
  auto poll_gives_up = [&]() -> bool {
    if (*status != 0) return true;
    if (global_ns() - t_start > PP.max_ns) {
      if (lane == 0) atomicExch((int*)PP.status, -6);
      return true;
    }
    const unsigned long long now = *progress;
    if (now != seen) {
      idle = 0;
      seen = now;
    } else if (++idle > PP.spin_limit) {
      if (lane == 0) atomicExch((int*)PP.status, -6);
      return true;
    } else {
      __nanosleep(256);
    }
    return false;
  };
  while (true) {
    if (*status != 0) return;  // whole warp: another warp gave up
    if (global_ns() - t_start > PP.max_ns) {
      if (lane == 0) atomicExch((int*)PP.status, -6);
      return;
    }
    // a member whose open phase has unclaimed items: the lanes look at 32 members at once,
    // starting from this warp's own member so that warps spread over the members
    int pick = -1;
    bool any_active = false;
    for (int j0 = 0; j0 < nact && pick < 0; j0 += 32) {
      const int j = j0 + lane;
      bool act = false, open = false;
      if (j < nact) {
        const PersistMember* m = PP.mem + (k0 + j) % nact;
        if (!*(volatile const int*)&m->finished) {
          act = true;
          const unsigned long long p = *(volatile const unsigned long long*)&m->phase;
          const int s = int(p % (N + 1));
          const long long ns = m->nstrips;
          const unsigned long long end = (p / (N + 1)) * (unsigned long long)(N * ns + 1) +
                                         (unsigned long long)s * ns + (s < N ? (unsigned long long)ns : 1ull);
          open = *(volatile const unsigned long long*)&m->ticket < end;
        }
      }
      any_active = __any_sync(kFull, act) || any_active;
      const unsigned b = __ballot_sync(kFull, open);
      if (b) pick = (k0 + j0 + __ffs(b) - 1) % nact;
    }
    if (!any_active) return;  // every member has finished
    if (pick < 0) {
      if (poll_gives_up()) return;
      continue;
    }
    // take the member's next ticket. Tickets number the member's work items in order: per
    // timestep N stage phases of nstrips items, then one finalize item. Warps that saw the
    // same open phase may take tickets past its end; such a ticket belongs to a later phase
    // and its warp waits for that phase to open (or drops it if the member finishes first)
    PersistMember* m = PP.mem + pick;
    const long long ns = m->nstrips;
    unsigned long long t = 0;
    if (lane == 0) t = atomicAdd(&m->ticket, 1ull);
    t = __shfl_sync(kFull, t, 0);
    const unsigned long long per = (unsigned long long)N * ns + 1;
    const unsigned long long r = t % per;
    const int s = r < (unsigned long long)N * ns ? int(r / ns) : N;
    const unsigned long long q = (t / per) * (N + 1) + s;  // the ticket's phase
    const unsigned long long nwork = s < N ? (unsigned long long)ns : 1ull;
    bool dropped = false, stop = false;
    while (*(volatile unsigned long long*)&m->phase < q) {
      if (*(volatile int*)&m->finished) {
        dropped = true;
        break;
      }
      if (poll_gives_up()) {
        stop = true;
        break;
      }
    }
    if (stop) return;
    if (dropped) continue;
    __threadfence();  // acquire: the previous phases' writes of every warp
    if (s < N) {
      // stage s, strip item r % ns: the member's parameters to shared memory, then the sweep
      static_assert(sizeof(StageParams<T>) % 4 == 0, "parameter block copied as 32-bit words");
      const unsigned* src = reinterpret_cast<const unsigned*>(PP.Ps + size_t(s) * nact + pick);
      unsigned* dst = reinterpret_cast<unsigned*>(&Psh[wib]);
      for (int i = lane; i < int(sizeof(StageParams<T>) / 4); i += 32) dst[i] = src[i];
      __syncwarp();
      // the member's interior strips (listed first) run the interior sweep
      const StageParams<T>& SP = Psh[wib];
      const long long item = (long long)(r % ns);
      if (SP.istrips && item < SP.n_istrips)
        sweep_strip_interior<T, kPersistRows, P2, EDDY, true>(SP, SP.istrips[item]);
      else if (SP.bstrips)
        sweep_strip<T, kPersistRows, P2, EDDY, true>(SP, SP.bstrips[item - SP.n_istrips]);
      else
        sweep_strip<T, kPersistRows, P2, EDDY, true>(SP, item);
      __syncwarp();
    } else {
      finalize_warp(PP.Fs[pick], red[wib]);
    }
    __threadfence();  // release this item's writes before counting it
    int last = 0;
    if (lane == 0) {
      last = atomicAdd(&m->done, 1u) + 1u == (unsigned)nwork;
      atomicAdd(PP.progress, 1ull);
    }
    last = __shfl_sync(kFull, last, 0);
    if (last) {
      __threadfence();  // acquire the other items of the phase
      if (lane == 0) {
        m->done = 0;
        // after a finalize the member goes on while its controller has a step running
        const bool more = s < N || (*(volatile int*)&PP.Fs[pick].ctl->done == 0);
        __threadfence();
        if (more) atomicExch(&m->phase, q + 1);
        else atomicExch(&m->finished, 1);
      }
      __syncwarp();
    }
    idle = 0;
    seen = *progress;
  }
}

#ifdef SV_DEFINE_COMMON_KERNELS
// Host-API accept (RungeKutta.hpp:428-431): flip the state parity, apply the pending tallies.
__global__ void accept_kernel(Ctl* ctl) {
  ctl->cur ^= 1;
  ctl->accepted++;
  ctl->rain_in += ctl->pend_rain;
  ctl->outflow += ctl->pend_out;
  ctl->wall_in += ctl->pend_wall;
  ctl->volume = ctl->pend_vol;
}
__global__ void begin_step_kernel(Ctl* ctl, int new_step, long long budget) {
  if (new_step) {
    ctl->t_local = 0.0;
    ctl->step_accepted = 0;
    ctl->step_repeated = 0;
  }
  ctl->done = 0;
  ctl->budget = budget;
}
// start a batched advance of queued steps: each member's first step (or, with no steps
// queued or a member that already failed, nothing: done at once)
__global__ void begin_queue_kernel(const FinalizeParams* Fs, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Ctl* c = Fs[i].ctl;
  StepQueue* q = Fs[i].q;
  c->t_local = 0.0;
  c->step_accepted = 0;
  c->step_repeated = 0;
  c->budget = q->limit;
  q->k = 0;
  q->status = 0;
  q->cur = c->cur;
  if (c->error) {
    q->status = -5;
    c->done = 1;
  } else if (q->n <= 0) {
    c->done = 1;
  } else {
    if (!q->keep_first) *Fs[i].fc = q->f[0];
    c->done = 0;
  }
}
// done flags of a batch into one array (1: step complete, nonzero error code: -1)
__global__ void gather_done_kernel(Ctl* const* ctls, int n, int* done) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  done[i] = ctls[i]->error ? -1 : ctls[i]->done;
}
#endif

// Volume of a cell field: per-CTA FP64 partials (same tiling and reduction as the stage
// kernel's last stage), then a fixed-order sum.
template <typename T, int TX, int TY>
__global__ void __launch_bounds__(TX * TY) volume_partials_kernel(const T* h, int nx, int ny, double area,
                                                                  double* part) {
  __shared__ double red[TX * TY / 32];
  const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
  const int gx = blockIdx.x * TX + tx, gy = blockIdx.y * TY + ty;
  double v = 0.0;
  if (gx < nx && gy < ny) v = double(h[(long long)gy * nx + gx]) * area;
  double s = block_sum<TX * TY>(v, red);
  if (threadIdx.x == 0) part[(long long)blockIdx.y * gridDim.x + blockIdx.x] = s;
}
template <int NT> __global__ void __launch_bounds__(NT) sum_kernel(const double* p, long long n, double* out) {
  __shared__ double red[NT];
  double r = fixed_sum<NT>(p, n, red);
  if (threadIdx.x == 0) *out = r;
}

// ------------------------------- debug / per-function kernels -------------------------
template <typename T> struct DebugParams {
  int nx, ny;
  double dx, dy;
  const T *h, *u, *v, *z;
  T *dhdx, *dudx, *dvdx, *dzdx, *dhdy, *dudy, *dvdy, *dzdy;
  T *fh, *fu, *fv, *fz, *fb;
};

// SpatialDerivativeOperationKernel over global arrays (State.cpp:187-192, Constants.cpp:39-40)
template <typename T> __global__ void debug_slopes_kernel(const DebugParams<T> D) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long n = (long long)D.nx * D.ny;
  if (i >= n) return;
  int gx = int(i % D.nx), gy = int(i / D.nx);
  bool hasW = gx > 0, hasE = gx < D.nx - 1, hasN = gy < D.ny - 1, hasS = gy > 0;
  Div<T> divx = mkdiv<T>(D.dx), divy = mkdiv<T>(D.dy);
  const T* src[4] = {D.h, D.u, D.v, D.z};
  T* dx_[4] = {D.dhdx, D.dudx, D.dvdx, D.dzdx};
  T* dy_[4] = {D.dhdy, D.dudy, D.dvdy, D.dzdy};
  for (int f = 0; f < 4; ++f) {
    const T* a = src[f];
    T c = a[i];
    T l = hasW ? a[i - 1] : c, r = hasE ? a[i + 1] : c;
    dx_[f][i] = minmod3<T>(l, hasW, c, hasE, r, divx);
    T nn = hasN ? a[i + D.nx] : c, ss = hasS ? a[i - D.nx] : c;
    dy_[f][i] = minmod3<T>(nn, hasN, c, hasS, ss, divy);
  }
}

// SaintVenantFluxKernel over all faces (Fluxes.cpp:55-64)
template <typename T> __global__ void debug_flux_kernel(const DebugParams<T> D) {
  long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long nvf = (long long)(D.nx + 1) * D.ny;
  long long nf = nvf + (long long)(D.ny + 1) * D.nx;
  if (f >= nf) return;
  auto cell = [&](long long i) {
    CellV<T> c;
    c.h = D.h[i]; c.u = D.u[i]; c.v = D.v[i]; c.z = D.z[i];
    c.dhdx = D.dhdx[i]; c.dudx = D.dudx[i]; c.dvdx = D.dvdx[i]; c.dzdx = D.dzdx[i];
    c.dhdy = D.dhdy[i]; c.dudy = D.dudy[i]; c.dvdy = D.dvdy[i]; c.dzdy = D.dzdy[i];
    return c;
  };
  FaceF<T> F;
  T br;
  if (f < nvf) {
    long long fx = f % (D.nx + 1), fy = f / (D.nx + 1);
    int edge = fx == 0 ? -1 : (fx == D.nx ? 1 : 0);
    long long l = fy * D.nx + (edge == -1 ? 0 : fx - 1);
    long long r = fy * D.nx + (edge == 1 ? D.nx - 1 : fx);
    br = face_flux<T, 0>(cell(l), cell(r), edge, T(0.5) * T(D.dx), mkdiv<T>(D.dx), F);
  } else {
    long long f2 = f - nvf;
    long long fx = f2 % D.nx, fy = f2 / D.nx;
    int edge = fy == 0 ? -1 : (fy == D.ny ? 1 : 0);
    long long l = (edge == -1 ? 0 : fy - 1) * D.nx + fx;
    long long r = (edge == 1 ? D.ny - 1 : fy) * D.nx + fx;
    br = face_flux<T, 1>(cell(l), cell(r), edge, T(0.5) * T(D.dy), mkdiv<T>(D.dy), F);
  }
  D.fh[f] = F.h; D.fu[f] = F.u; D.fv[f] = F.v; D.fz[f] = F.z; D.fb[f] = br;
}

// temporal derivative + sources + boundaries per cell from the global face arrays
template <typename T>
__global__ void debug_cell_kernel(const StageParams<T> P, const DebugParams<T> D, T* nh, T* sf) {
  long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long n = (long long)P.nx * P.ny;
  if (g >= n) return;
  const Ctl* ctl = P.ctl;
  const double dt_d = ctl->dt;
  int gx = int(g % P.nx), gy = int(g / P.nx);
  CellCtx<T> c;
  c.divx = mkdiv<T>(P.dx); c.divy = mkdiv<T>(P.dy);
  c.divdt = mkdiv<T>(dt_d); c.divL = mkdiv<T>(P.L);
  c.dt = T(dt_d); c.dt_d = dt_d; c.tsub_d = ctl->t_local + P.c_s * dt_d;
  c.manning = P.manning; c.rain_mode = P.rain_mode; c.head_first = P.head_first;
  long long w = (long long)gy * (P.nx + 1) + gx, e = w + 1;
  long long sf_ = (long long)(P.nx + 1) * P.ny + (long long)gy * P.nx + gx, nf_ = sf_ + P.nx;
  FaceF<T> fw{D.fh[w], D.fu[w], D.fv[w], D.fz[w]}, fe{D.fh[e], D.fu[e], D.fv[e], D.fz[e]};
  FaceF<T> fs{D.fh[sf_], D.fu[sf_], D.fv[sf_], D.fz[sf_]}, fn{D.fh[nf_], D.fu[nf_], D.fv[nf_], D.fz[nf_]};
  const DevForcing fc = *P.fc;
  T kh, ku, kv;
  double rain, removed, wall;
  EddyIn<T> ed{};
  if (P.eddy) {  // second derivatives from the mesh-wide slope fields
    const int nx = P.nx;
    const bool hasW = gx > 0, hasE = gx < nx - 1, hasN = gy < P.ny - 1, hasS = gy > 0;
    ed.ux = D.dudx[g]; ed.uy = D.dudy[g]; ed.vx = D.dvdx[g]; ed.vy = D.dvdy[g];
    ed.uxx = minmod3<T>(hasW ? D.dudx[g - 1] : ed.ux, hasW, ed.ux, hasE, hasE ? D.dudx[g + 1] : ed.ux, c.divx);
    ed.vxx = minmod3<T>(hasW ? D.dvdx[g - 1] : ed.vx, hasW, ed.vx, hasE, hasE ? D.dvdx[g + 1] : ed.vx, c.divx);
    ed.uyy = minmod3<T>(hasN ? D.dudy[g + nx] : ed.uy, hasN, ed.uy, hasS, hasS ? D.dudy[g - nx] : ed.uy, c.divy);
    ed.vyy = minmod3<T>(hasN ? D.dvdy[g + nx] : ed.vy, hasN, ed.vy, hasS, hasS ? D.dvdy[g - nx] : ed.vy, c.divy);
  }
  cell_dudt<T, CellCtx<T>, true>(P, fc, c, g, gx, gy, D.h[g], D.u[g], D.v[g], D.dhdx[g], D.dhdy[g], D.dzdx[g],
                                 D.dzdy[g], fw, fe, fs, fn, kh, ku, kv, rain, removed, wall, nh + g, sf + g, &ed);
  P.Kout[0][g] = kh; P.Kout[1][g] = ku; P.Kout[2][g] = kv;
}

}  // namespace svk
