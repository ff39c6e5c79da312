// sv_pow43.h -- x^(4/3) for the Manning friction slope, identical bit for bit on
// the host (g++, -ffp-contract=off) and on the device (nvcc, explicit _rn intrinsics).
//
// The reference evaluates Sf = n^2 |V| pow(inv_h, 4/3) with sycl::pow
// (src/SaintVenant/SourceTerms/ManningRoughnessSourceTerm.cpp:64-65). sycl::pow is
// not correctly rounded (SYCL allows 16 ulp) and differs between a CPU libm and a GPU
// libdevice, so two faithful implementations of that line cannot agree bit for bit.
// This project therefore uses one routine, written here from the mathematics, on both
// sides of every FP64 parity comparison:
//
//   x = m * 2^e  (m in [0.5, 1), exact bit split)
//   e = 3q + r   (r in {0, 1, 2}),  w = m * 2^r in [0.5, 4)
//   y0 = cubic least-squares fit of w^(-1/3) on [0.5, 4)   (relative error < 4e-2)
//   three Newton steps for the inverse cube root  y <- y + y (1 - w y^3) / 3
//   c = w y^2 (= w^(1/3)), then one Newton correction  c <- c - (c^3 - w) y^2 / 3
//   x^(4/3) = x * (c * 2^q)
//
// Only IEEE-754 +, -, * (each correctly rounded, no fused multiply-add) and exact exponent
// scaling are used -- no division and no library call -- so the result depends on nothing
// but the operation order written below, and costs about 36 FP64 operations.
// Accuracy: within 1.7 ulp of the exact x^(4/3) over [1e-7, 1e3] (measured against an
// 80-bit evaluation); it differs from glibc pow(x, 4.0/3.0) by at most 12 ulp there,
// mostly because 4.0/3.0 itself is rounded in the reference's exponent.
#pragma once

#if defined(__CUDACC__)
#define SV_HD __host__ __device__ __forceinline__
#else
#define SV_HD inline
#endif

#if defined(__CUDA_ARCH__)
#define SVP_MUL(a, b) __dmul_rn((a), (b))
#define SVP_ADD(a, b) __dadd_rn((a), (b))
#define SVP_SUB(a, b) __dsub_rn((a), (b))
#define SVP_DIV(a, b) __ddiv_rn((a), (b))
#else
#include <cmath>
#define SVP_MUL(a, b) ((a) * (b))
#define SVP_ADD(a, b) ((a) + (b))
#define SVP_SUB(a, b) ((a) - (b))
#define SVP_DIV(a, b) ((a) / (b))
#endif

namespace sv_math {

// Least-squares cubic for w^(-1/3), w in [0.5, 4), relative error 3.96e-2.
constexpr double kRcbrtSeed3 = -0.019273;
constexpr double kRcbrtSeed2 = 0.18161161;
constexpr double kRcbrtSeed1 = -0.63413856;
constexpr double kRcbrtSeed0 = 1.48409885;
constexpr double kThird = 1.0 / 3.0;

SV_HD double pow43(double x) {
  // NaN, +-0, +inf and negative inputs: the Manning term only calls this for
  // h > 1e-6, i.e. x > 0; everything else is passed through unchanged
  // (NaN stays NaN, inf stays inf).
  if (!(x > 0.0) || !(x < 1.0e300)) return x;
  int e;
#if defined(__CUDA_ARCH__)
  double m = frexp(x, &e);
#else
  double m = std::frexp(x, &e);
#endif
  // floor division of e by 3 (e may be negative)
  int q = (e >= 0) ? (e / 3) : -((-e + 2) / 3);
  int r = e - 3 * q;
  double w = m;
  if (r == 1) w = SVP_MUL(m, 2.0);
  else if (r == 2) w = SVP_MUL(m, 4.0);
  double y = SVP_ADD(SVP_MUL(SVP_ADD(SVP_MUL(SVP_ADD(SVP_MUL(kRcbrtSeed3, w), kRcbrtSeed2), w),
                                     kRcbrtSeed1), w), kRcbrtSeed0);
  for (int it = 0; it < 3; ++it) {
    double y3 = SVP_MUL(SVP_MUL(y, y), y);
    y = SVP_ADD(y, SVP_MUL(SVP_MUL(y, SVP_SUB(1.0, SVP_MUL(w, y3))), kThird));
  }
  double cb = SVP_MUL(SVP_MUL(w, y), y);
  double res = SVP_SUB(SVP_MUL(SVP_MUL(cb, cb), cb), w);
  cb = SVP_SUB(cb, SVP_MUL(res, SVP_MUL(SVP_MUL(y, y), kThird)));
#if defined(__CUDA_ARCH__)
  double c = ldexp(cb, q);
#else
  double c = std::ldexp(cb, q);
#endif
  return SVP_MUL(x, c);
}

}  // namespace sv_math
