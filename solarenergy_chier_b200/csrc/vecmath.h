// Small float3 toolkit shared by the host scene code and the sm_100a kernels.
//
// Every helper evaluates its expression in the same order as the reference's
// vector helpers (Util/vector_arithmetic.cuh: dot left-to-right, cross in
// x,y,z order, normalize as v * (1/len), reflect as i - (2n)*dot(n,i)), so
// host geometry built here is bit-identical to the reference's host build
// when both are compiled without FMA contraction (-ffp-contract=off).
// The reciprocal square root inside normalize is the correctly rounded
// 1/sqrt(x): on the host it is evaluated in double and rounded once to float,
// which reproduces the host rsqrtf that the reference's nvcc build links
// into its scene code (checked output-for-output on 1.2e8 inputs across 61
// binades); on the device it equals __frsqrt_rn, the round-to-nearest rsqrt
// (computed by qm_rsqrt_series below, bit-identical to it).  So
// host geometry equals the reference's host geometry bit for bit and device
// normalisation equals the CPU oracle's, instead of following the hardware
// approximation.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

#if defined(__CUDACC__)
#define QM_HD __host__ __device__ __forceinline__
#else
#define QM_HD inline
#endif

namespace qm {
// Reference tolerance (Util/global_constant.h:11).  It is a double literal in
// the reference, so every comparison against it happens in double precision.
constexpr double kEps = 1e-5;
}  // namespace qm

// A float compared with the double 1e-5, decided in float.  1e-5f is the
// largest float below 1e-5 (9.99999974737875e-06; the next float,
// 1.0000000656873453e-05, lies above it) and no float equals 1e-5, so for
// every float x (NaN included):
//   (double)x <  1e-5  <=>  (double)x <= 1e-5  <=>  x <= 1e-5f
//   (double)x > -1e-5  <=>  (double)x >= -1e-5  <=>  x >= -1e-5f
//   (double)x < -1e-5  <=>  x < -1e-5f
// which saves the float-to-double conversions on the device.
QM_HD bool qm_below_eps(float x) { return x <= 1.0e-5f; }         // (double)x < 1e-5
QM_HD bool qm_above_neg_eps(float x) { return x >= -1.0e-5f; }    // (double)x > -1e-5
QM_HD bool qm_below_neg_eps(float x) { return x < -1.0e-5f; }     // (double)x < -1e-5

// Explicitly rounded float operations: on the device the _rn intrinsics,
// which the compiler never fuses; on the host plain operators (host code is
// built with -ffp-contract=off).
QM_HD float qm_rn_add(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fadd_rn(a, b);
#else
  return a + b;
#endif
}
QM_HD float qm_rn_sub(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fsub_rn(a, b);
#else
  return a - b;
#endif
}
QM_HD float qm_rn_mul(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fmul_rn(a, b);
#else
  return a * b;
#endif
}
QM_HD float qm_rn_div(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fdiv_rn(a, b);
#else
  return a / b;
#endif
}

#if defined(__CUDACC__)
// Correctly rounded 1/sqrt(x) for x in [2^-125, 2^125), from the hardware
// estimate y (rsqrt.approx, relative error below 2^-22) refined by the series
// 1/sqrt(x) = y (1 - e)^(-1/2) = y (1 + e/2 + 3e^2/8 + O(e^3)), e = 1 - x y^2.
// The product x y is split without error into h + eh (the FMA two-product),
// so e = (1 - h y) - eh y carries one rounding of a number below 2^-21, and
// the last FMA rounds y + y (e/2 + 3e^2/8) once.  It equals __frsqrt_rn on
// every float (checked exhaustively on the B200: qmcrt_debug_check_primitives);
// inputs outside the range (zero, subnormal, huge, negative, inf, NaN) take
// __frsqrt_rn itself.  About 9 instructions against __frsqrt_rn's ~28.
// (The device-only helpers here are declared for nvcc's host pass too, with
// bodies only in the device pass.)
__device__ __forceinline__ float qm_rsqrt_series(float x) {
#if defined(__CUDA_ARCH__)
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  const float h = __fmul_rn(x, y);
  const float eh = __fmaf_rn(x, y, -h);
  const float t = __fmaf_rn(-h, y, 1.0f);
  const float e = __fmaf_rn(-eh, y, t);
  const float c = __fmul_rn(e, __fmaf_rn(0.375f, e, 0.5f));
  return __fmaf_rn(y, c, y);
#else
  return x;
#endif
}
#endif

// Correctly rounded reciprocal square root 1/sqrt(x): on the device the
// series refinement above (bit-identical to __frsqrt_rn); on the host
// evaluated in double and rounded once to float.
QM_HD float qm_rn_rsqrt(float x) {
#if defined(__CUDA_ARCH__)
  if (__float_as_uint(x) - 0x01000000u < 0x7c000000u) return qm_rsqrt_series(x);  // x in [2^-125, 2^125)
  return __frsqrt_rn(x);
#else
  return (float)(1.0 / sqrt((double)x));
#endif
}
// The same value for arguments known to lie in [2^-125, 2^125) or to be NaN
// (the squared length of a unit-scale vector): the series without the range
// test, whose branch costs the tracer about 1.3 % of its time per call site.
QM_HD float qm_rn_rsqrt_unit(float x) {
#if defined(__CUDA_ARCH__)
  return qm_rsqrt_series(x);
#else
  return (float)(1.0 / sqrt((double)x));
#endif
}
// a / b rounded to nearest, given y = RN(1/b) (b and y normal): Markstein's
// division -- q = RN(a y) lies within one ulp of a/b, so r = a - b q is
// exact (one FMA) and RN(q + r y) = RN(a/b) (Muller et al., Handbook of
// Floating-Point Arithmetic, Markstein's theorem) -- wherever the remainder
// stays normal (a and a/b in [2^-90, 2^90] suffices).  Below that the result
// is a tiny number that may differ from RN(a/b) in its last places; where
// RN(a y) overflows, it is RN(a y) itself
// (an infinity of the right sign; RN(q + r y) would be NaN there).  Three
// instructions against __fdiv_rn's ~16; callers state why those two regimes
// cannot change their results.
QM_HD float qm_div_by_rcp(float a, float b, float y) {
#if defined(__CUDA_ARCH__)
  const float q = __fmul_rn(a, y);
  const float r = __fmaf_rn(-b, q, a);
  const float q1 = __fmaf_rn(r, y, q);
  return fabsf(q) < INFINITY ? q1 : q;
#else
  (void)y;
  return a / b;
#endif
}

#if defined(__CUDACC__)
// 1/x rounded to nearest for |x| in [2^-100, 2^100]: the hardware estimate
// (rcp.approx) and one Newton step y + y (1 - x y) by FMA.  Equal to
// __frcp_rn on every such x (checked exhaustively on the B200).
__device__ __forceinline__ float qm_rcp_newton(float x) {
#if defined(__CUDA_ARCH__)
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return __fmaf_rn(__fmaf_rn(-x, y, 1.0f), y, y);
#else
  return 1.0f / x;
#endif
}
// a / b by Markstein's division given y = RN(1/b), for a, b and a/b in the
// normal range with the remainder a - b q normal too (|a| in [2^-60, 2^70)
// and |b| in [2^-50, 2^64) suffice): equal to __fdiv_rn there (Markstein's
// theorem, as for qm_div_by_rcp).
__device__ __forceinline__ float qm_div_markstein(float a, float b, float y) {
  const float q = __fmul_rn(a, y);
  return __fmaf_rn(__fmaf_rn(-b, q, a), y, q);
}
// sqrt(x) rounded to nearest from y = RN(1/sqrt(x)), for x in [2^-100, 2^126):
// s = RN(x y), the remainder x - s^2 is exact by FMA, and RN(s + (x - s^2) y/2)
// is the correctly rounded root (Markstein's square-root iteration; equal to
// __fsqrt_rn on every such x, checked exhaustively).
__device__ __forceinline__ float qm_sqrt_by_rsqrt(float x, float y) {
  const float s = __fmul_rn(x, y);
  return __fmaf_rn(__fmaf_rn(-s, s, x), __fmul_rn(0.5f, y), s);
}
#endif

// Approximate forms (device: the hardware reciprocal square root and the
// reciprocal-multiply division, within 2 ulp for the magnitudes the tracer
// meets; host: the plain operations).
QM_HD float qm_fast_rsqrt(float x) {
#if defined(__CUDA_ARCH__)
  return rsqrtf(x);
#else
  return (float)(1.0 / sqrt((double)x));
#endif
}
QM_HD float qm_fast_div(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fdividef(a, b);
#else
  return a / b;
#endif
}

// Orthonormal frame aligned with a normal: the columns (u, n, v) map local
// (x, y, z) to world (shared by the three variants below).
namespace qm_frame {
struct Frame {
  float3 u, n, v;
  bool identity;
};
}  // namespace qm_frame

#define QA(a, b) ((a) + (b))
#define QS(a, b) ((a) - (b))
#define QM(a, b) ((a) * (b))
#define QD(a, b) ((a) / (b))
#define QR(x) qm_rn_rsqrt(x)
#define QRU(x) qm_rn_rsqrt(x)
namespace qm {
#include "vecmath_impl.h"
}  // namespace qm
#undef QA
#undef QS
#undef QM
#undef QD
#undef QR
#undef QRU

#define QA(a, b) qm_rn_add((a), (b))
#define QS(a, b) qm_rn_sub((a), (b))
#define QM(a, b) qm_rn_mul((a), (b))
#define QD(a, b) qm_rn_div((a), (b))
#define QR(x) qm_rn_rsqrt(x)
#define QRU(x) qm_rn_rsqrt_unit(x)
namespace qs {
using qm::kEps;
#include "vecmath_impl.h"
}  // namespace qs
#undef QA
#undef QS
#undef QM
#undef QD
#undef QR
#undef QRU

#define QA(a, b) ((a) + (b))
#define QS(a, b) ((a) - (b))
#define QM(a, b) ((a) * (b))
#define QD(a, b) qm_fast_div((a), (b))
#define QR(x) qm_fast_rsqrt(x)
#define QRU(x) qm_fast_rsqrt(x)
namespace qf {
using qm::kEps;
#include "vecmath_impl.h"
}  // namespace qf
#undef QA
#undef QS
#undef QM
#undef QD
#undef QR
#undef QRU
