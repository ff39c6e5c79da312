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
  return (__double2hiint(x) & 0x7ff00000) != 0x7ff00000;
}
__device__ __forceinline__ bool finite_(float x) {
  return (__float_as_int(x) & 0x7f800000) != 0x7f800000;
}

// Bit-pattern helpers: magnitude comparisons, NaN tests and absolute values on the integer
// pipe (for non-negative, non-NaN IEEE values the bit patterns order like the numbers).
template <typename T> struct Bits;
template <> struct Bits<double> {
  using I = long long;
  static constexpr I kMag = 0x7fffffffffffffffLL, kInf = 0x7ff0000000000000LL, kSign = (I)0x8000000000000000ULL;
  __device__ static I of(double x) { return __double_as_longlong(x); }
  __device__ static double from(I i) { return __longlong_as_double(i); }
};
template <> struct Bits<float> {
  using I = int;
  static constexpr I kMag = 0x7fffffff, kInf = 0x7f800000, kSign = (I)0x80000000u;
  __device__ static I of(float x) { return __float_as_int(x); }
  __device__ static float from(I i) { return __int_as_float(i); }
};
// For doubles the tests work on the 32-bit halves (the integer pipe has no 64-bit compare).
__device__ __forceinline__ bool isnan_b(double x) {
  unsigned hi = unsigned(__double2hiint(x)) & 0x7fffffffu;
  return hi > 0x7ff00000u || (hi == 0x7ff00000u && __double2loint(x) != 0);
}
__device__ __forceinline__ bool isnan_b(float x) { return (__float_as_int(x) & 0x7fffffff) > 0x7f800000; }
__device__ __forceinline__ double abs_b(double x) {
  return __hiloint2double(__double2hiint(x) & 0x7fffffff, __double2loint(x));
}
__device__ __forceinline__ float abs_b(float x) { return __int_as_float(__float_as_int(x) & 0x7fffffff); }
__device__ __forceinline__ bool iszero_b(double x) {
  return ((__double2hiint(x) & 0x7fffffff) | __double2loint(x)) == 0;
}
__device__ __forceinline__ bool iszero_b(float x) { return (__float_as_int(x) & 0x7fffffff) == 0; }
// fmax(x, 0) up to the sign of a zero result: 0 for negative or NaN x
__device__ __forceinline__ double max0_b(double x) { return (__double2hiint(x) < 0 || isnan_b(x)) ? 0.0 : x; }
__device__ __forceinline__ float max0_b(float x) {
  int i = __float_as_int(x);
  return (i < 0 || (i & 0x7fffffff) > 0x7f800000) ? 0.0f : x;
}
// The reference's minmod pair T(0.5) * (sign(a) + sign(b)) * min(|a|, |b|) for non-NaN a, b:
// +min when both are positive, -min when both are negative, a zero otherwise.
__device__ __forceinline__ double mm2(double a, double b) {
  const int ha = __double2hiint(a), hb = __double2hiint(b);
  const bool nz = !iszero_b(a) && !iszero_b(b);
  const double m = fmin(abs_b(a), abs_b(b));
  const bool same = (ha ^ hb) >= 0;
  return (same && nz) ? (ha < 0 ? -m : m) : 0.0;
}
__device__ __forceinline__ float mm2(float a, float b) {
  const int ia = __float_as_int(a), ib = __float_as_int(b);
  const bool nz = (ia & 0x7fffffff) != 0 && (ib & 0x7fffffff) != 0;
  const float m = fminf(abs_b(a), abs_b(b));
  return ((ia ^ ib) >= 0 && nz) ? (ia < 0 ? -m : m) : 0.0f;
}

// sycl::sign: 1, -1, +-0 for +-0, 0 for NaN
template <typename T> __device__ __forceinline__ T ssign(T x) {
  return x > T(0) ? T(1) : (x < T(0) ? T(-1) : (x == x ? x : T(0)));
}
// sign(f) != sign(u) for an f with |f| > |u| (so f is neither zero nor NaN, and u is not
// NaN): u is a zero, or the two have opposite signs. The same truth value as comparing the
// sycl::sign results, without forming them.
template <typename T> __device__ __forceinline__ bool opposes(T f, T u) {
  return u == T(0) || ((f < T(0)) != (u < T(0)));
}
// sycl::min(x, y): y if y < x, else x
template <typename T> __device__ __forceinline__ T smin(T x, T y) { return (y < x) ? y : x; }
// fmax: IEEE maxNum
__device__ __forceinline__ double sfmax(double x, double y) { return fmax(x, y); }
__device__ __forceinline__ float sfmax(float x, float y) { return fmaxf(x, y); }
__device__ __forceinline__ double sfmin(double x, double y) { return fmin(x, y); }
__device__ __forceinline__ float sfmin(float x, float y) { return fminf(x, y); }
__device__ __forceinline__ double ssqrt(double x) { return sqrt(x); }
// FP32 path: the hardware's approximate square root (sqrt.approx, a relative error of a few
// ulp) instead of the correctly rounded one; 0, infinity and NaN pass through, subnormal
// arguments (depths below 1e-39 m, speeds below 1e-19 m/s) count as 0. The FP32 path is held
// to a depth tolerance, not to bit parity. The arguments here are never negative.
__device__ __forceinline__ float ssqrt(float x) {
  float r;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ double sfabs(double x) { return fabs(x); }
__device__ __forceinline__ float sfabs(float x) { return fabsf(x); }

// b + t*0 as in the reference's tangential terms: b, or NaN when t is not finite
template <typename T> __device__ __forceinline__ T add_tangential(T b, T t) {
  return finite_(t) ? b : Lim<T>::nan();
}
// Same for t = hd * s without forming the product: for |s| < 2^1000 and hd < 2^20 the
// product is finite; beyond that (or for a non-finite s) the product decides.
__device__ __forceinline__ double add_tangential_s(double b, double hd, double s) {
  const unsigned e = (unsigned(__double2hiint(s)) >> 20) & 0x7ffu;
  if (e < 1023u + 1000u) return b;
  return finite_(hd * s) ? b : Lim<double>::nan();
}
__device__ __forceinline__ float add_tangential_s(float b, float hd, float s) {
  return finite_(hd * s) ? b : Lim<float>::nan();
}

// Out-of-line IEEE division: the rare operands outside the range where the correction below
// is exact (zero, subnormal, huge, inf, NaN). Kept out of line so the common path is not
// predicated with a full division sequence.
static __device__ __noinline__ double div_slow(double x, double d) { return x / d; }

// Division by a launch-constant divisor d with rd = RN(1/d).
struct DivD {
  double d, rd;
  __device__ __forceinline__ double operator()(double x) const {
    const unsigned e = (unsigned(__double2hiint(x)) >> 20) & 0x7ffu;  // biased exponent
    if (e - (1023u - 900u) > 1800u) return div_slow(x, d);         // outside [2^-900, 2^901)
    double q0 = x * rd;
    double r = fma(-q0, d, x);
    return fma(r, rd, q0);
  }
};
// Division by a power of two d = 2^k: x * 2^-k is the same real number as x / 2^k, so the
// two round identically (subnormal, zero, inf and NaN results included): one multiply.
struct DivP2 {
  double rd;
  __device__ __forceinline__ double operator()(double x) const { return x * rd; }
};
// FP32 path (not held to bit parity): multiply by the rounded reciprocal.
struct DivF {
  float rd;
  __device__ __forceinline__ float operator()(float x) const { return x * rd; }
};
template <typename T> struct DivC;
template <> struct DivC<double> { using type = DivD; };
template <> struct DivC<float> { using type = DivF; };
template <typename T> using Div = typename DivC<T>::type;
// divider for the mesh spacing: exact power-of-two multiply when P2, else the general one
template <typename T, bool P2> struct DivXC { using type = Div<T>; };
template <> struct DivXC<double, true> { using type = DivP2; };
template <typename T, bool P2> using DivX = typename DivXC<T, P2>::type;

__device__ __forceinline__ DivD make_div(double d) { return DivD{d, 1.0 / d}; }
__device__ __forceinline__ DivF make_divf(float d) { return DivF{1.0f / d}; }

// ---------------------------------------------------------------------------------------
// Minmod3 slope, theta = 2 (src/SpatialDerivative/Minmod3.hpp:22-84) on a uniform axis of
// spacing d: hasL / hasR say whether the left / right neighbour exists (the missing side
// has dx = 0 and U = U_c, src/Mesh/Cartesian2DMesh.hpp:477-519). The reference's
// theta*(a-b)/d and (r-l)/(2d) are formed as 2*((a-b)/d) and ((r-l)/d)*0.5, which are
// exact power-of-two rescalings of the same correctly rounded quotient.
// ---------------------------------------------------------------------------------------
// Minmod3 from the difference quotients of a uniform axis: qL = (Uc-Ul)/d, qR = (Ur-Uc)/d,
// qC = (Ur-Ul)/d. Two-sided: lhs = 2 qL, rhs = 2 qR, central = qC/2; one-sided: the missing
// difference is NaN and the central difference uses U_l = U_c, so central = the present
// quotient. The pair minmods follow Minmod3.hpp:66-80 including the NaN rules (a NaN outer
// difference returns the central one; a NaN central one gives sign(outer)/2 * |outer|).
template <typename T>
__device__ __forceinline__ T minmod3q(T qL, bool hasL, T qR, bool hasR, T qC) {
  T outer, central;
  if (hasL && hasR) {
    T lhs = T(2) * qL, rhs = T(2) * qR;
    central = qC * T(0.5);
    outer = isnan_b(lhs) ? rhs : (isnan_b(rhs) ? lhs : mm2(lhs, rhs));
  } else if (hasR) {
    outer = T(2) * qR;
    central = qR;
  } else if (hasL) {
    outer = T(2) * qL;
    central = qL;
  } else {
    return T(0);
  }
  if (isnan_b(outer)) return central;
  if (isnan_b(central)) return T(0.5) * outer;
  return mm2(outer, central);
}

template <typename T, typename DV>
__device__ __forceinline__ T minmod3(T Ul, bool hasL, T Uc, bool hasR, T Ur, const DV& div) {
  T qL = hasL ? div(Uc - Ul) : T(0);
  T qR = hasR ? div(Ur - Uc) : T(0);
  T qC = (hasL && hasR) ? div(Ur - Ul) : T(0);
  return minmod3q<T>(qL, hasL, qR, hasR, qC);
}

// Cell values and slopes needed by a face.
template <typename T> struct CellV {
  T h, u, v, z;
  T dhdx, dudx, dvdx, dzdx, dhdy, dudy, dvdy, dzdy;
};
template <typename T> struct FaceF { T h, u, v, z; };

// One side of a face after the MUSCL reconstruction (FluxKernel.cpp:161-187): bed, depth and
// the normal and tangential velocity components at the face.
template <typename T> struct Side { T zb, h, un, ut; };

// b + hd * n on the face side of the left cell (recon_m) or b - hd * n on that of the right
// cell (recon_p), plus the tangential term hd * t * 0 as a finiteness test (TCHK; without it
// the term is dropped, which only changes results whose slopes are not finite).
template <typename T, bool TCHK> __device__ __forceinline__ T recon_m(T b, T hd, T n, T t) {
  const T r = b + hd * n;
  if constexpr (TCHK) return add_tangential_s(r, hd, t);
  return r;
}
template <typename T, bool TCHK> __device__ __forceinline__ T recon_p(T b, T hd, T n, T t) {
  const T r = b - hd * n;
  if constexpr (TCHK) return add_tangential_s(r, hd, t);
  return r;
}

// The face sides of a cell with both neighbours along DIR in the mesh and a valid bed (no edge
// or coded-out masks apply): as the left cell of its face in +DIR (side_m) and as the right
// cell of its face in -DIR (side_p).
template <typename T, int DIR, bool TCHK>
__device__ __forceinline__ Side<T> side_m(const CellV<T>& c, T hd) {
  if constexpr (DIR == 0)
    return {recon_m<T, TCHK>(c.z, hd, c.dzdx, c.dzdy), recon_m<T, TCHK>(c.h, hd, c.dhdx, c.dhdy),
            recon_m<T, TCHK>(c.u, hd, c.dudx, c.dudy), recon_m<T, TCHK>(c.v, hd, c.dvdx, c.dvdy)};
  else
    return {recon_m<T, TCHK>(c.z, hd, c.dzdy, c.dzdx), recon_m<T, TCHK>(c.h, hd, c.dhdy, c.dhdx),
            recon_m<T, TCHK>(c.v, hd, c.dvdy, c.dvdx), recon_m<T, TCHK>(c.u, hd, c.dudy, c.dudx)};
}
template <typename T, int DIR, bool TCHK>
__device__ __forceinline__ Side<T> side_p(const CellV<T>& c, T hd) {
  if constexpr (DIR == 0)
    return {recon_p<T, TCHK>(c.z, hd, c.dzdx, c.dzdy), recon_p<T, TCHK>(c.h, hd, c.dhdx, c.dhdy),
            recon_p<T, TCHK>(c.u, hd, c.dudx, c.dudy), recon_p<T, TCHK>(c.v, hd, c.dvdx, c.dvdy)};
  else
    return {recon_p<T, TCHK>(c.z, hd, c.dzdy, c.dzdx), recon_p<T, TCHK>(c.h, hd, c.dhdy, c.dhdx),
            recon_p<T, TCHK>(c.v, hd, c.dvdy, c.dvdx), recon_p<T, TCHK>(c.u, hd, c.dudy, c.dudx)};
}

// The flux of a face from its two reconstructed sides (FluxKernel.cpp:189-291): the face bed,
// the wet/dry branch and the Rusanov-type fluxes of h, the normal and the tangential momentum,
// and the bed-step (z) term. Returns the branch code (1, 2.25, 2.75, 3 or 4).
// TCHK = false drops the tangential finiteness terms (u_t * 0, g h * 0), which only matter
// when a side's value is not finite (the FP32 interior sweeps; a non-finite state).
template <typename T, int DIR, bool TCHK = true, typename DV>
__device__ __forceinline__ T face_combine(Side<T> m, Side<T> p, const DV& divd, FaceF<T>& F) {
  const T g = T(kG);
  const T zb_m = m.zb, zb_p = p.zb, un_m = m.un, un_p = p.un, ut_m = m.ut, ut_p = p.ut;
  T h_m = m.h, h_p = p.h;
  T zb_f = sfmax(zb_m, zb_p);
  T y_m = zb_m + h_m;
  T y_p = zb_p + h_p;
  h_m = max0_b(h_m);
  h_p = max0_b(h_p);
  // momentum components: normal gets 0.5*spd and the +-g*h term; tangential gets
  // 1.0*spd and a g*h*0 term (NaN only for infinite h).
  // The reference's branch chain (FluxKernel.cpp:208-289): 1 if both levels are above the
  // face bed, else 2 if both are at or below it, else 3 if the left one is above, else 4.
  // With a NaN level neither comparison holds, which selects branch 4.
  const bool both = (y_m > zb_f) && (y_p > zb_f);
  const bool dry2 = !both && (y_m <= zb_f) && (y_p <= zb_f);
  const bool wm = !both && !dry2 && (y_m > zb_f);  // branch 3: left side only
  T branch;
  T Fn, Ft;
  if (!dry2) {
    // Branches 1 (both sides above the face bed), 3 (left only) and 4 (right only)
    // evaluated without divergence: each side's terms, then the branch's own combination of
    // them selected per face.
    const T c_m = ssqrt(g * h_m), c_p = ssqrt(g * h_p);
    const T spd_m = TCHK ? add_tangential(un_m, ut_m) : un_m;
    const T spd_p = TCHK ? add_tangential(un_p, ut_p) : un_p;
    const T hf_m = h_m * spd_m, hf_p = h_p * spd_p;
    const T gh_m = g * h_m, gh_p = g * h_p;
    const T nf_m = un_m * (T(0.5) * spd_m) + gh_m;
    const T nf_p = both ? un_p * (T(0.5) * spd_p) - gh_p : un_p * (T(0.5) * spd_p) + gh_p;
    const T tf_m = TCHK ? add_tangential(ut_m * spd_m, gh_m) : ut_m * spd_m;
    const T tf_p = TCHK ? add_tangential(ut_p * spd_p, gh_p) : ut_p * spd_p;
    // |spd + sign(spd) c| = |spd| + c, or 0 when spd is an exact zero (sign(0) = 0)
    const T a_m = iszero_b(spd_m) ? T(0) : abs_b(spd_m) + c_m;
    const T a_p = iszero_b(spd_p) ? T(0) : abs_b(spd_p) + c_p;
    const T a = both ? sfmax(a_p, a_m) : (wm ? a_m : a_p);
    const T ha = T(0.5) * a;
    const T Sh = both ? hf_p + hf_m : (wm ? hf_m : hf_p);
    const T Dh = both ? h_p - h_m : (wm ? -h_m : h_p);
    const T Sn = both ? nf_p + nf_m : (wm ? nf_m : nf_p);
    const T Dn = both ? un_p - un_m : (wm ? -un_m : un_p);
    const T St = both ? tf_p + tf_m : (wm ? tf_m : tf_p);
    const T Dt = both ? ut_p - ut_m : (wm ? -ut_m : ut_p);
    F.h = T(0.5) * Sh - ha * Dh;
    Fn = T(0.5) * Sn - ha * Dn;
    Ft = T(0.5) * St - ha * Dt;
    F.z = both ? (zb_m - zb_p) * g : divd(wm ? h_p : h_m);
    branch = both ? T(1) : (wm ? T(3) : T(4));
  } else {
    // branch 2: both water levels at or below the face bed (FluxKernel.cpp:235-254)
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
  }
  if (DIR == 0) { F.u = Fn; F.v = Ft; }
  else { F.u = Ft; F.v = Fn; }
  return branch;
}

// ---------------------------------------------------------------------------------------
// SaintVenantFluxKernel::operator() (src/SaintVenant/FluxKernel.cpp:62-295) for one face
// of direction DIR (0: vertical face, flow along x; 1: horizontal face, flow along y).
// L / R are the cells from get_adjacent_cells (equal on the mesh edge), edge is -1/0/+1.
// d = dx or dy; hd = 0.5*d. Returns the branch code (1, 2.25, 2.75, 3, 4, or 0 when the
// face borders coded-out cells).
// ---------------------------------------------------------------------------------------
template <typename T, int DIR, typename DV>
__device__ __forceinline__ T face_flux(CellV<T> L, CellV<T> R, int edge, T hd, const DV& divd, FaceF<T>& F) {
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
  const Side<T> m{recon_m<T, true>(zb_L, hd, dzn_L, dzt_L), recon_m<T, true>(h_L, hd, dhn_L, dht_L),
                  recon_m<T, true>(un_L, hd, dunn_L, dunt_L), recon_m<T, true>(ut_L, hd, dutn_L, dutt_L)};
  const Side<T> p{recon_p<T, true>(zb_R, hd, dzn_R, dzt_R), recon_p<T, true>(h_R, hd, dhn_R, dht_R),
                  recon_p<T, true>(un_R, hd, dunn_R, dunt_R), recon_p<T, true>(ut_R, hd, dutn_R, dutt_R)};
  return face_combine<T, DIR>(m, p, divd, F);
}

// Per-launch scalars of one stage evaluation (update_dUdt arguments and forcing).
template <typename T, typename DX = Div<T>> struct CellCtx {
  DX divx, divy;
  Div<T> divdt, divL;
  T dt;          // timestep (TT=double for T=double)
  double dt_d, tsub_d;
  int manning, rain_mode, head_first;
};

// Depth-rate of the discharge boundary (DischargeBoundarySourceTerm.cpp:47-66) for
// boundary values q0, q1 at depth h; returns 0 when the cell is skipped.
template <typename T, typename CC>
__device__ __forceinline__ T discharge_rate(T q0, T q1, T h, const CC& c, bool& applied) {
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
template <typename T, typename CC>
__device__ __forceinline__ T head_target(T h0, T h1, const CC& c) {
  T dhb = c.divL(h1 - h0);
  T hnow = h0 + T(c.tsub_d) * dhb;
  T hnext = hnow + c.dt * dhb;
  T target = T(0.5) * (hnow + hnext);
  if (target <= T(0)) target = T(0);
  return target;
}

// Manning friction (ManningRoughnessSourceTerm.cpp:53-87): adds to du, dv.
__device__ __forceinline__ double pow43_(double x) { return sv_math::pow43(x); }
// FP32 path: x^(4/3) = 2^(4/3 log2 x) on the special-function unit (relative error about
// 1e-6 over the range of 1/h here); 0 gives 0, infinity infinity, NaN NaN.
__device__ __forceinline__ float pow43_(float x) { return __powf(x, 4.0f / 3.0f); }
// h / (h^2 + 1e-3) of the roughness term: IEEE division in FP64, the fast reciprocal form
// in FP32
__device__ __forceinline__ double manning_inv_h(double h) { return h / (h * h + 1e-3); }
__device__ __forceinline__ float manning_inv_h(float h) { return __fdividef(h, h * h + 1e-3f); }

// Roughness term (ManningRoughnessSourceTerm.cpp): the increments fu, fv of du/dt, dv/dt;
// false (no increment) on cells of 1e-6 m depth or less.
template <typename T, typename CC>
__device__ __forceinline__ bool manning_term(T h, T u, T v, T ns, T nd, T ds, T dd, const CC& c, T& fu, T& fv,
                                             T* n_out, T* sf_out) {
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
    T inv_h = manning_inv_h(h);
    T sf = n * n * ssqrt(u * u + v * v) * pow43_(inv_h);
    if (sf_out) *sf_out = sf;
    fu = -T(kG) * sf * u;
    fv = -T(kG) * sf * v;
    T fudt = fu * c.dt, fvdt = fv * c.dt;
    if (sfabs(fudt) > sfabs(u) && opposes(fudt, u)) fu = -c.divdt(u);
    if (sfabs(fvdt) > sfabs(v) && opposes(fvdt, v)) fv = -c.divdt(v);
    return true;
  }
  if (sf_out) *sf_out = T(0);
  return false;
}
template <typename T, typename CC>
__device__ __forceinline__ void manning_apply(T h, T u, T v, T ns, T nd, T ds, T dd, const CC& c,
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
    T inv_h = manning_inv_h(h);
    T sf = n * n * ssqrt(u * u + v * v) * pow43_(inv_h);
    if (sf_out) *sf_out = sf;
    T fu = -T(kG) * sf * u;
    T fv = -T(kG) * sf * v;
    T fudt = fu * c.dt, fvdt = fv * c.dt;
    if (sfabs(fudt) > sfabs(u) && opposes(fudt, u)) fu = -c.divdt(u);
    if (sfabs(fvdt) > sfabs(v) && opposes(fvdt, v)) fv = -c.divdt(v);
    du = du + fu;
    dv = dv + fv;
  } else if (sf_out) {
    *sf_out = T(0);
  }
}

// Energy loss (EnergyLossSourceTerm.cpp:64-87): du = -0.5 u fx |U|, dv = -0.5 v fy |U| on
// cells deeper than 1e-6 m, capped like the roughness term.
template <typename T, typename CC>
__device__ __forceinline__ bool energy_loss_term(T h, T u, T v, T fx, T fy, const CC& c, T& eu, T& ev) {
  if (!(h > T(1e-6))) return false;
  T hyp = ssqrt(u * u + v * v);
  eu = T(-0.5) * u * fx * hyp;
  ev = T(-0.5) * v * fy * hyp;
  T eudt = eu * c.dt, evdt = ev * c.dt;
  if (sfabs(eudt) > sfabs(u) && opposes(eudt, u)) eu = -c.divdt(u);
  if (sfabs(evdt) > sfabs(v) && opposes(evdt, v)) ev = -c.divdt(v);
  return true;
}
template <typename T, typename CC>
__device__ __forceinline__ void energy_loss_apply(T h, T u, T v, T fx, T fy, const CC& c, T& du, T& dv) {
  if (!(h > T(1e-6))) return;
  T hyp = ssqrt(u * u + v * v);
  T eu = T(-0.5) * u * fx * hyp;
  T ev = T(-0.5) * v * fy * hyp;
  T eudt = eu * c.dt, evdt = ev * c.dt;
  if (sfabs(eudt) > sfabs(u) && opposes(eudt, u)) eu = -c.divdt(u);
  if (sfabs(evdt) > sfabs(v) && opposes(evdt, v)) ev = -c.divdt(v);
  du = du + eu;
  dv = dv + ev;
}

// Inputs of the eddy-viscosity term at one cell: the stage's first slopes of u and v and
// their second derivatives (Minmod3 of the slopes along the same axis,
// EddyViscositySourceTerm.hpp:222-228).
template <typename T> struct EddyIn {
  T ux, uy, vx, vy;      // du/dx, du/dy, dv/dx, dv/dy
  T uxx, uyy, vxx, vyy;  // d2u/dx2, d2u/dy2, d2v/dx2, d2v/dy2
};
// Smagorinsky coefficient (SmagorinskyCoefficientKernel, EddyViscositySourceTerm.cpp:97-110):
// mu_c + mu_s * area * sqrt(u_x^2 + v_y^2 + 0.5 (|u_y| + |v_x|)^2), the square taken as a
// product (the reference's pow(x, 2))
template <typename T>
__device__ __forceinline__ T smagorinsky_mu(T mc, T ms, T area, const EddyIn<T>& e) {
  const T a = sfabs(e.uy) + sfabs(e.vx);
  return mc + ms * area * ssqrt(e.ux * e.ux + e.vy * e.vy + T(0.5) * (a * a));
}
// Eddy viscosity (EddyViscositySourceKernel, EddyViscositySourceTerm.cpp:46-78):
// du = -mu (u_xx + u_yy), dv = -mu (v_xx + v_yy) on cells deeper than 1e-6 m, capped like the
// roughness term.
template <typename T, typename CC>
__device__ __forceinline__ bool eddy_term(T h, T u, T v, T mu, const EddyIn<T>& e, const CC& c, T& fu, T& fv) {
  if (!(h > T(1e-6))) return false;
  fu = -mu * (e.uxx + e.uyy);
  fv = -mu * (e.vxx + e.vyy);
  T fudt = fu * c.dt, fvdt = fv * c.dt;
  if (sfabs(fudt) > sfabs(u) && opposes(fudt, u)) fu = -c.divdt(u);
  if (sfabs(fvdt) > sfabs(v) && opposes(fvdt, v)) fv = -c.divdt(v);
  return true;
}

// Infiltration (InfiltrationSourceTerm.cpp:43-62): the depth taken this evaluation,
// rate * dt limited by the water present and by the remaining soil capacity.
template <typename T, typename CC>
__device__ __forceinline__ T infiltration_depth(T h, T rate, T cap, const CC& c) {
  T dh = rate * c.dt;
  if (dh > h) dh = h;
  if (dh > cap) dh = cap;
  return dh;
}

}  // namespace svd
