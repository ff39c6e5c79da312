// sv_device.cuh -- per-face and per-cell arithmetic of the Saint-Venant step on sm_100a.
//
// Every function here evaluates one reference kernel body for one face or one cell,
// in registers, so the fused stage kernel and the per-function debug kernels share one
// definition. For T = double the translation unit is compiled with -fmad=false: each
// + - * / is a separately rounded IEEE operation in the reference's order, so results are
// bit-identical to the reference arithmetic at T = double. Two rewrites are exact and are
// used for speed:
//   * x / d for a divisor d fixed per launch (dx, dy, dt, L) is computed by Markstein's
//     correction q = fma(fma(-x*rd, d, x), rd, x*rd) with rd = RN(1/d); this is the
//     correctly rounded quotient for |x| in [2^-900, 2^900) (a fall-back division covers
//     the rest), i.e. bit-identical to x / d.
//   * a term t * 0 added to a value b (the reference's tangential reconstruction terms,
//     `... * ydir` with ydir == 0) equals b unless t is not finite, where it is NaN; it is
//     applied as that test instead of a multiply and an add (the sign of an exact zero may
//     differ, which never changes a non-zero result).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "sv_pow43.h"

namespace svd {

constexpr double kG = 9.81;

template <typename T> struct Lim;
template <> struct Lim<double> {
  __device__ static double nan() { return __longlong_as_double(0x7ff8000000000000LL); }
};
template <> struct Lim<float> {
  __device__ static float nan() { return __int_as_float(0x7fc00000); }
};

__device__ __forceinline__ bool finite_(double x) {
  return (__double_as_longlong(x) & 0x7ff0000000000000LL) != 0x7ff0000000000000LL;
}
__device__ __forceinline__ bool finite_(float x) {
  return (__float_as_int(x) & 0x7f800000) != 0x7f800000;
}

// sycl::sign: 1, -1, +-0 for +-0, 0 for NaN
template <typename T> __device__ __forceinline__ T ssign(T x) {
  return x > T(0) ? T(1) : (x < T(0) ? T(-1) : (x == x ? x : T(0)));
}
// sycl::min(x, y): y if y < x, else x
template <typename T> __device__ __forceinline__ T smin(T x, T y) { return (y < x) ? y : x; }
// fmax: IEEE maxNum
__device__ __forceinline__ double sfmax(double x, double y) { return fmax(x, y); }
__device__ __forceinline__ float sfmax(float x, float y) { return fmaxf(x, y); }
__device__ __forceinline__ double sfmin(double x, double y) { return fmin(x, y); }
__device__ __forceinline__ float sfmin(float x, float y) { return fminf(x, y); }
__device__ __forceinline__ double ssqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float ssqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double sfabs(double x) { return fabs(x); }
__device__ __forceinline__ float sfabs(float x) { return fabsf(x); }

// b + t*0 as in the reference's tangential terms: b, or NaN when t is not finite
template <typename T> __device__ __forceinline__ T add_tangential(T b, T t) {
  return finite_(t) ? b : Lim<T>::nan();
}

// Division by a launch-constant divisor d with rd = RN(1/d).
struct DivD {
  double d, rd;
  __device__ __forceinline__ double operator()(double x) const {
    long long e = (__double_as_longlong(x) >> 52) & 0x7ff;  // biased exponent
    if (e < 1023 - 900 || e > 1023 + 900) return x / d;     // zero, tiny, huge, inf, NaN
    double q0 = x * rd;
    double r = fma(-q0, d, x);
    return fma(r, rd, q0);
  }
};
struct DivF {
  float d, rd;
  __device__ __forceinline__ float operator()(float x) const { return __fdiv_rn(x, d); }
};
template <typename T> struct DivC;
template <> struct DivC<double> { using type = DivD; };
template <> struct DivC<float> { using type = DivF; };
template <typename T> using Div = typename DivC<T>::type;

__device__ __forceinline__ DivD make_div(double d) { return DivD{d, 1.0 / d}; }
__device__ __forceinline__ DivF make_divf(float d) { return DivF{d, 1.0f / d}; }

// ---------------------------------------------------------------------------------------
// Minmod3 slope, theta = 2 (src/SpatialDerivative/Minmod3.hpp:22-84) on a uniform axis of
// spacing d: hasL / hasR say whether the left / right neighbour exists (the missing side
// has dx = 0 and U = U_c, src/Mesh/Cartesian2DMesh.hpp:477-519). The reference's
// theta*(a-b)/d and (r-l)/(2d) are formed as 2*((a-b)/d) and ((r-l)/d)*0.5, which are
// exact power-of-two rescalings of the same correctly rounded quotient.
// ---------------------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T minmod3(T Ul, bool hasL, T Uc, bool hasR, T Ur, const Div<T>& div) {
  T outer, central;
  if (hasL && hasR) {
    T lhs = T(2) * div(Uc - Ul);
    T rhs = T(2) * div(Ur - Uc);
    central = div(Ur - Ul) * T(0.5);
    if (lhs != lhs) outer = rhs;
    else if (rhs != rhs) outer = lhs;
    else outer = T(0.5) * (ssign(lhs) + ssign(rhs)) * smin(sfabs(lhs), sfabs(rhs));
  } else if (hasR) {  // west/north edge: lhs difference undefined
    outer = T(2) * div(Ur - Uc);
    central = div(Ur - Uc);
  } else if (hasL) {
    outer = T(2) * div(Uc - Ul);
    central = div(Uc - Ul);
  } else {
    return T(0);
  }
  if (outer != outer) return central;
  return T(0.5) * (ssign(outer) + ssign(central)) * smin(sfabs(outer), sfabs(central));
}

// Cell values and slopes needed by a face.
template <typename T> struct CellV {
  T h, u, v, z;
  T dhdx, dudx, dvdx, dzdx, dhdy, dudy, dvdy, dzdy;
};
template <typename T> struct FaceF { T h, u, v, z; };

// ---------------------------------------------------------------------------------------
// SaintVenantFluxKernel::operator() (src/SaintVenant/FluxKernel.cpp:62-295) for one face
// of direction DIR (0: vertical face, flow along x; 1: horizontal face, flow along y).
// L / R are the cells from get_adjacent_cells (equal on the mesh edge), edge is -1/0/+1.
// d = dx or dy; hd = 0.5*d. Returns the branch code (1, 2.25, 2.75, 3, 4, or 0 when the
// face borders coded-out cells).
// ---------------------------------------------------------------------------------------
template <typename T, int DIR>
__device__ __forceinline__ T face_flux(CellV<T> L, CellV<T> R, int edge, T hd, const Div<T>& divd,
                                       FaceF<T>& F) {
  const T g = T(kG);
  const T zb_L0 = L.z, zb_R0 = R.z;
  T zb_L = zb_L0, zb_R = zb_R0;
  // coded-out cells (NaN bed), FluxKernel.cpp:83-107
  if (zb_L0 != zb_L0) {
    L = R;
    if (edge == 1) { F.h = F.u = F.v = F.z = T(0); return T(0); }
    edge = -1;
  }
  if (zb_R0 != zb_R0) {
    if (edge == -1) { F.h = F.u = F.v = F.z = T(0); return T(0); }
    R = L;
    edge = 1;
  }
  const bool mL = edge < 0, mR = edge > 0;
  // edge/coded-out masks, FluxKernel.cpp:111-148 (x*0 only where the mask applies)
  T h_L = mL ? L.h * T(0) : L.h;
  T h_R = mR ? R.h * T(0) : R.h;
  // normal velocity is masked, tangential is not
  T un_L = DIR == 0 ? L.u : L.v, un_R = DIR == 0 ? R.u : R.v;
  T ut_L = DIR == 0 ? L.v : L.u, ut_R = DIR == 0 ? R.v : R.u;
  if (mL) un_L = un_L * T(0);
  if (mR) un_R = un_R * T(0);
  // slopes: normal (along DIR) and tangential
  T dhn_L = DIR == 0 ? L.dhdx : L.dhdy, dht_L = DIR == 0 ? L.dhdy : L.dhdx;
  T dhn_R = DIR == 0 ? R.dhdx : R.dhdy, dht_R = DIR == 0 ? R.dhdy : R.dhdx;
  T dzn_L = DIR == 0 ? L.dzdx : L.dzdy, dzt_L = DIR == 0 ? L.dzdy : L.dzdx;
  T dzn_R = DIR == 0 ? R.dzdx : R.dzdy, dzt_R = DIR == 0 ? R.dzdy : R.dzdx;
  // slopes of the normal velocity component (masked with it)
  T dunn_L = DIR == 0 ? L.dudx : L.dvdy, dunt_L = DIR == 0 ? L.dudy : L.dvdx;
  T dunn_R = DIR == 0 ? R.dudx : R.dvdy, dunt_R = DIR == 0 ? R.dudy : R.dvdx;
  // slopes of the tangential velocity component (not masked)
  T dutn_L = DIR == 0 ? L.dvdx : L.dudy, dutt_L = DIR == 0 ? L.dvdy : L.dudx;
  T dutn_R = DIR == 0 ? R.dvdx : R.dudy, dutt_R = DIR == 0 ? R.dvdy : R.dudx;
  if (mL) {
    dhn_L = dhn_L * T(0); dht_L = dht_L * T(0); dzn_L = dzn_L * T(0); dzt_L = dzt_L * T(0);
    dunn_L = dunn_L * T(0); dunt_L = dunt_L * T(0);
  }
  if (mR) {
    dhn_R = dhn_R * T(0); dht_R = dht_R * T(0); dzn_R = dzn_R * T(0); dzt_R = dzt_R * T(0);
    dunn_R = dunn_R * T(0); dunt_R = dunt_R * T(0);
  }
  // walls for coded-out / edge cells, FluxKernel.cpp:152-157
  if (mL) zb_L = zb_R + h_R * T(2);
  if (mR) zb_R = zb_L + h_L * T(2);
  // MUSCL reconstruction, FluxKernel.cpp:161-187. For DIR 0 the reference adds the
  // normal term then the tangential (*0) term; for DIR 1 the tangential term first. Both
  // orders give b + n (a finite exact zero never changes a non-zero sum).
  T zb_m = add_tangential(zb_L + hd * dzn_L, hd * dzt_L);
  T h_m = add_tangential(h_L + hd * dhn_L, hd * dht_L);
  T un_m = add_tangential(un_L + hd * dunn_L, hd * dunt_L);
  T ut_m = add_tangential(ut_L + hd * dutn_L, hd * dutt_L);
  T zb_p = add_tangential(zb_R - hd * dzn_R, hd * dzt_R);
  T h_p = add_tangential(h_R - hd * dhn_R, hd * dht_R);
  T un_p = add_tangential(un_R - hd * dunn_R, hd * dunt_R);
  T ut_p = add_tangential(ut_R - hd * dutn_R, hd * dutt_R);

  T zb_f = sfmax(zb_m, zb_p);
  T y_m = zb_m + h_m;
  T y_p = zb_p + h_p;
  h_m = sfmax(h_m, T(0));
  h_p = sfmax(h_p, T(0));
  // momentum components: normal gets 0.5*spd and the +-g*h term; tangential gets
  // 1.0*spd and a g*h*0 term (NaN only for infinite h).
  T branch;
  T Fn, Ft;
  if (y_m > zb_f && y_p > zb_f) {
    branch = T(1);
    T c_m = ssqrt(g * h_m), c_p = ssqrt(g * h_p);
    T spd_m = add_tangential(un_m, ut_m), spd_p = add_tangential(un_p, ut_p);
    T hf_m = h_m * spd_m, hf_p = h_p * spd_p;
    T gh_m = g * h_m, gh_p = g * h_p;
    T nf_m = un_m * (T(0.5) * spd_m) + gh_m;
    T nf_p = un_p * (T(0.5) * spd_p) - gh_p;
    T tf_m = add_tangential(ut_m * spd_m, gh_m);
    T tf_p = add_tangential(ut_p * spd_p, gh_p);
    T a = sfmax(sfabs(spd_p + ssign(spd_p) * c_p), sfabs(spd_m + ssign(spd_m) * c_m));
    T ha = T(0.5) * a;
    F.h = T(0.5) * (hf_p + hf_m) - ha * (h_p - h_m);
    Fn = T(0.5) * (nf_p + nf_m) - ha * (un_p - un_m);
    Ft = T(0.5) * (tf_p + tf_m) - ha * (ut_p - ut_m);
    F.z = (zb_m - zb_p) * g;
  } else if (y_m <= zb_f && y_p <= zb_f) {
    F.h = T(0);
    if (zb_p > zb_m) {
      branch = T(2.25);
      T gh = g * h_m;
      Fn = T(0.5) * gh;
      Ft = T(0.5) * (gh * T(0));
      F.z = -h_m * T(0.5) * g;
    } else {
      branch = T(2.75);
      T gh = g * h_p;
      Fn = T(-0.5) * gh;
      Ft = T(-0.5) * (gh * T(0));
      F.z = h_p * T(0.5) * g;
    }
  } else if (y_m > zb_f) {
    branch = T(3);
    T c_m = ssqrt(g * h_m);
    T spd_m = add_tangential(un_m, ut_m);
    T hf_m = h_m * spd_m;
    T gh_m = g * h_m;
    T nf_m = un_m * (T(0.5) * spd_m) + gh_m;
    T tf_m = add_tangential(ut_m * spd_m, gh_m);
    T a = sfabs(spd_m + ssign(spd_m) * c_m);
    T ha = T(0.5) * a;
    F.h = T(0.5) * hf_m - ha * (-h_m);
    Fn = T(0.5) * nf_m - ha * (-un_m);
    Ft = T(0.5) * tf_m - ha * (-ut_m);
    F.z = divd(h_p);
  } else {
    branch = T(4);
    T c_p = ssqrt(g * h_p);
    T spd_p = add_tangential(un_p, ut_p);
    T hf_p = h_p * spd_p;
    T gh_p = g * h_p;
    T nf_p = un_p * (T(0.5) * spd_p) + gh_p;
    T tf_p = add_tangential(ut_p * spd_p, gh_p);
    T a = sfabs(spd_p + ssign(spd_p) * c_p);
    T ha = T(0.5) * a;
    F.h = T(0.5) * hf_p - ha * h_p;
    Fn = T(0.5) * nf_p - ha * un_p;
    Ft = T(0.5) * tf_p - ha * ut_p;
    F.z = divd(h_m);
  }
  if (DIR == 0) { F.u = Fn; F.v = Ft; }
  else { F.u = Ft; F.v = Fn; }
  return branch;
}

// Per-launch scalars of one stage evaluation (update_dUdt arguments and forcing).
template <typename T> struct CellCtx {
  Div<T> divx, divy, divdt, divL;
  T dt;          // timestep (TT=double for T=double)
  double dt_d, tsub_d;
  int manning, rain_mode, head_first;
};

// Depth-rate of the discharge boundary (DischargeBoundarySourceTerm.cpp:47-66) for
// boundary values q0, q1 at depth h; returns 0 when the cell is skipped.
template <typename T>
__device__ __forceinline__ T discharge_rate(T q0, T q1, T h, const CellCtx<T>& c, bool& applied) {
  applied = false;
  if (q0 != T(0) || q1 != T(0)) {
    applied = true;
    T dqdt = c.divL(q1 - q0);
    T qnow = q0 + T(c.tsub_d) * dqdt;
    T qnext = qnow + c.dt * dqdt;
    T dh = T(0.5) * (qnow + qnext);
    bool clamp = c.rain_mode == 0 ? (h - dh * c.dt <= T(0)) : (h + dh * c.dt <= T(0));
    if (clamp) dh = -c.divdt(h);
    return dh;
  }
  return T(0);
}

// HeadBoundarySourceKernel (HeadBoundarySourceTerm.cpp:47-65): target depth for the
// boundary values h0, h1; the caller assigns dhdt = (target - h) / dt.
template <typename T>
__device__ __forceinline__ T head_target(T h0, T h1, const CellCtx<T>& c) {
  T dhb = c.divL(h1 - h0);
  T hnow = h0 + T(c.tsub_d) * dhb;
  T hnext = hnow + c.dt * dhb;
  T target = T(0.5) * (hnow + hnext);
  if (target <= T(0)) target = T(0);
  return target;
}

// Manning friction (ManningRoughnessSourceTerm.cpp:53-87): adds to du, dv.
__device__ __forceinline__ double pow43_(double x) { return sv_math::pow43(x); }
__device__ __forceinline__ float pow43_(float x) { return x * cbrtf(x); }

template <typename T>
__device__ __forceinline__ void manning_apply(T h, T u, T v, T ns, T nd, T ds, T dd, const CellCtx<T>& c,
                                              T& du, T& dv, T* n_out, T* sf_out) {
  T n;
  if (ns == nd) {
    n = ns;  // mix(n, n, t) = n + 0*t = n: t = smoothstep(...) is always finite
  } else {
    T t = sfmin(sfmax((h - ds) / (dd - ds), T(0)), T(1));
    T ss = t * t * (T(3) - T(2) * t);
    n = ns + (nd - ns) * ss;
  }
  if (n_out) *n_out = n;
  if (h > T(1e-6)) {
    T inv_h = h / (h * h + T(1e-3));
    T sf = n * n * ssqrt(u * u + v * v) * pow43_(inv_h);
    if (sf_out) *sf_out = sf;
    T fu = -T(kG) * sf * u;
    T fv = -T(kG) * sf * v;
    T fudt = fu * c.dt, fvdt = fv * c.dt;
    if (sfabs(fudt) > sfabs(u) && ssign(fudt) != ssign(u)) fu = -c.divdt(u);
    if (sfabs(fvdt) > sfabs(v) && ssign(fvdt) != ssign(v)) fv = -c.divdt(v);
    du = du + fu;
    dv = dv + fv;
  } else if (sf_out) {
    *sf_out = T(0);
  }
}

}  // namespace svd
