// Device geometry of one ray outside the grid walk, shared by the tracer
// (tracer.cu) and the differentiable forward / adjoint (diff.cu): the
// micro-facet of a task, the receiver intersections and the task lookup.
// Every operation is explicitly rounded (qs::), so results do not depend on
// the unit's FMA contraction setting and equal the CPU oracle's.
#pragma once

#include <climits>

#include "device_scene.h"
#include "vecmath.h"

namespace qm {

__device__ __forceinline__ float3 xyz(float4 v) { return make_float3(v.x, v.y, v.z); }

// CylinderReceiver::GIntersect (Scene/DataStructure/Receiver/CylinderReceiver.cuh:39-89),
// every operation explicitly rounded: delta = |Ro|^2 - tp^2 cancels
// catastrophically for far heliostats (|Ro|^2 ~ 5e5 m^2, float spacing
// 0.03 m^2), so a fused multiply-add there would move rays across the
// cylinder's silhouette relative to the reference's rounding.
// acos takes its argument clamped to [-1, 1]; the reference prints an error
// and lets a NaN through when rounding pushes it outside.
__device__ __forceinline__ bool cylinder_hit(const DevReceiver& r, float3 o, float3 d, float& t, float& u, float& v) {
  float2 l = make_float2(qm_rn_sub(o.x, r.pos.x), qm_rn_sub(o.z, r.pos.z));
  const float r2 = qm_rn_mul(r.size.x, r.size.x);
  if (qs::dot2(l, l) <= r2) return false;
  float2 ro = make_float2(qm_rn_sub(r.pos.x, o.x), qm_rn_sub(r.pos.z, o.z));
  // The horizontal direction's squared length D, its correctly rounded
  // 1/sqrt and sqrt (normalize2 and length2 of the reference's test): for
  // D in [2^-100, 2^125) -- every ray but a vertical one -- from the series
  // rsqrt, the root by Markstein's iteration from it and later the division
  // by it by Markstein's method, each equal to CUDA's correctly rounded
  // operation there; otherwise by those operations themselves.
  const float2 dxz = make_float2(d.x, d.z);
  const float D = qs::dot2(dxz, dxz);
  const bool regular = __float_as_uint(D) - 0x0d800000u < 0x70800000u;
  float tp, len;
  if (regular) {
    const float inv = qm_rsqrt_series(D);
    tp = qs::dot2(ro, make_float2(qm_rn_mul(dxz.x, inv), qm_rn_mul(dxz.y, inv)));
    len = qm_sqrt_by_rsqrt(D, inv);
  } else {
    tp = qs::dot2(ro, qs::normalize2(dxz));
    len = sqrtf(D);
  }
  float delta = qm_rn_sub(qs::dot2(ro, ro), qm_rn_mul(tp, tp));
  if (qm_below_neg_eps(tp) || delta > r2) return false;
  float t_plus = delta <= 0.0f ? r.size.x : sqrtf(qm_rn_sub(r2, delta));
  const float num = qm_rn_sub(tp, t_plus);
  // |num| in [2^-60, 2^70) (a distance from 1e-18 m to 1e21 m) and len in
  // [2^-50, 2^63): Markstein's conditions hold
  if (regular && __float_as_uint(fabsf(num)) - 0x21800000u < 0x41000000u)
    t = qm_div_markstein(num, len, qm_rcp_newton(len));
  else
    t = qm_rn_div(num, len);
  float3 ip = qs::add(qs::mul(d, t), o);
  // (ip.y - pos.y) / height by Markstein's division with the host's RN(1/height):
  // equal to the correctly rounded quotient wherever it and the numerator lie
  // in [2^-90, 2^90]; below that u rounds to 0.5 either way, and where the
  // product overflows u is infinite (a miss) either way.
  u = qm_rn_add(qm_div_by_rcp(qm_rn_sub(ip.y, r.pos.y), r.size.y, r.rcp_height), 0.5f);
  if (u < 0.0f || u > 1.0f) return false;
  float2 cs = qs::normalize2(make_float2(qm_rn_sub(ip.x, r.pos.x), qm_rn_sub(ip.z, r.pos.z)));
  float cx = fminf(fmaxf(cs.x, -1.0f), 1.0f);
#if defined(QM_TRACE_FAST_DIVIDE)
  // The double product with the reciprocal of 2 pi lies within one double
  // ulp of the quotient; rounded to float, the two agree on every float in
  // [0, pi] (all checked by tests/test_primitives_math.py), so this equals the
  // reference's acosf(x) / (2 * M_PI) for the same arc cosine.
  v = (float)((double)acosf(cx) * (1.0 / (2 * M_PI)));
#elif defined(QM_EXACT_ACOS)
  // The exact build evaluates the arc cosine in double and rounds it once
  // to float: the correctly rounded value, which the host C library's float
  // acosf (what the reference's host build and the CPU oracle call; glibc
  // 2.39 on this image) returns for all but 0.25 % of the floats in
  // [-1, 1].  The device's own acosf differs from the host's far more often
  // (about 4 hits in a million landed one column over at the benchmark
  // field); through the double evaluation about 6 in 10^8 do.
  v = (float)__ddiv_rn((double)(float)acos((double)cx), 2 * M_PI);
#else
  v = (float)__ddiv_rn((double)acosf(cx), 2 * M_PI);
#endif
  if (cs.y < 0) v = qm_rn_sub(1.0f, v);
  return true;
}

__device__ __forceinline__ bool receiver_hit(const DevReceiver& r, float3 o, float3 d, float& t, float& u, float& v) {
  if (r.type == 0) return qs::ray_parallelogram(o, d, r.a, r.ab, r.ac, t, u, v);
  return cylinder_hit(r, o, d, t, u, v);
}

// The cylinder test with every decision rounded as the reference rounds it
// and the arithmetic after the decisions approximated (the
// receiver-approximate production build): the inside test, tp and the
// silhouette test delta > r^2 -- which cancels catastrophically for far
// heliostats, so its last bits decide hits -- are explicitly rounded as in
// cylinder_hit; the distance t, the hit point and its (u, v) use FMA
// contraction, the hardware reciprocal square root and reciprocal-multiply
// divisions.  A hit can land one pixel over when (u, v) lies within a few
// ulp of a pixel edge; the u range test flips only for hits within about a
// micrometre of the image's first or last row.
__device__ __forceinline__ bool cylinder_hit_rx(const DevReceiver& r, float3 o, float3 d, float& t, float& u,
                                                float& v) {
  float2 l = make_float2(qm_rn_sub(o.x, r.pos.x), qm_rn_sub(o.z, r.pos.z));
  const float r2 = qm_rn_mul(r.size.x, r.size.x);
  if (qs::dot2(l, l) <= r2) return false;
  float2 ro = make_float2(qm_rn_sub(r.pos.x, o.x), qm_rn_sub(r.pos.z, o.z));
  const float dd = qm_rn_add(qm_rn_mul(d.x, d.x), qm_rn_mul(d.z, d.z));
  const float il = qm_rn_rsqrt(dd);
  const float tp = qs::dot2(ro, make_float2(qm_rn_mul(d.x, il), qm_rn_mul(d.z, il)));
  const float delta = qm_rn_sub(qs::dot2(ro, ro), qm_rn_mul(tp, tp));
  if (qm_below_neg_eps(tp) || delta > r2) return false;
  const float s = r2 - delta;
  const float t_plus = delta <= 0.0f ? r.size.x : (s > 0.0f ? s * rsqrtf(s) : 0.0f);
  t = (tp - t_plus) * il;
  const float3 ip = make_float3(d.x * t + o.x, d.y * t + o.y, d.z * t + o.z);
  u = __fdividef(ip.y - r.pos.y, r.size.y) + 0.5f;
  if (u < 0.0f || u > 1.0f) return false;
  const float ex = ip.x - r.pos.x, ez = ip.z - r.pos.z;
  const float cx = fminf(fmaxf(ex * rsqrtf(ex * ex + ez * ez), -1.0f), 1.0f);
  v = acosf(cx) * 0.15915494f;
  if (ez < 0) v = 1.0f - v;
  return true;
}

__device__ __forceinline__ bool receiver_hit_rx(const DevReceiver& r, float3 o, float3 d, float& t, float& u,
                                                float& v) {
  if (r.type == 0) return qs::ray_parallelogram(o, d, r.a, r.ab, r.ac, t, u, v);
  return cylinder_hit_rx(r, o, d, t, u, v);
}

// The same cylinder test in approximate arithmetic (the approximate-math
// tracer build): FMA contraction, the hardware reciprocal square root and
// reciprocal-multiply divisions, v scaled by a float 1/(2 pi).  Rays near a
// pixel boundary or at the cylinder's silhouette (where delta cancels) can
// round to the neighbouring pixel or the other side of the silhouette; the
// tracer's tests measure how many.
__device__ __forceinline__ bool cylinder_hit_approx(const DevReceiver& r, float3 o, float3 d, float& t, float& u,
                                                    float& v) {
  const float lx = o.x - r.pos.x, lz = o.z - r.pos.z;
  const float r2 = r.size.x * r.size.x;
  if (lx * lx + lz * lz <= r2) return false;
  const float dd = d.x * d.x + d.z * d.z;
  const float il = rsqrtf(dd);
  const float tp = -(lx * d.x + lz * d.z) * il;
  const float delta = (lx * lx + lz * lz) - tp * tp;
  if (qm_below_neg_eps(tp) || delta > r2) return false;
  const float s = r2 - delta;  // >= 0 here; 0 for a ray grazing the silhouette
  const float t_plus = delta <= 0.0f ? r.size.x : (s > 0.0f ? s * rsqrtf(s) : 0.0f);
  t = (tp - t_plus) * il;
  const float3 ip = make_float3(d.x * t + o.x, d.y * t + o.y, d.z * t + o.z);
  u = __fdividef(ip.y - r.pos.y, r.size.y) + 0.5f;
  if (u < 0.0f || u > 1.0f) return false;
  const float ex = ip.x - r.pos.x, ez = ip.z - r.pos.z;
  const float cx = fminf(fmaxf(ex * rsqrtf(ex * ex + ez * ez), -1.0f), 1.0f);
  v = acosf(cx) * 0.15915494f;
  if (ez < 0) v = 1.0f - v;
  return true;
}

__device__ __forceinline__ bool receiver_hit_approx(const DevReceiver& r, float3 o, float3 d, float& t, float& u,
                                                    float& v) {
  if (r.type == 0) return qf::ray_parallelogram(o, d, r.a, r.ab, r.ac, t, u, v);
  return cylinder_hit_approx(r, o, d, t, u, v);
}

// Micro-facet centres and normals (rectangle_heliostat::map_microhelio_center_and_normal,
// Scene/DataStructure/Heliostat/RectangleHelio.cu:54-80; focusFlatRectangle_heliostat
// kernels, FocusFlatRectangleHelio.cu:12-64), evaluated per facet instead of
// materialised; explicitly rounded.
//
// Micro-facet f in its heliostat's local frame: its centre (the point the
// heliostat frame turns into world space) and, for focus-flat heliostats,
// the local normal of its sub-heliostat (flat facets share the heliostat
// normal).  Returns true for focus-flat.
__device__ __forceinline__ bool facet_local(const DevTask& T, int f, float3& local, float3& local_normal) {
  const int per_row = T.row_col.y * T.sub_row_col.y;
  int row = f / per_row;
  int col = f % per_row;
  const float px = T.pixel_length;
  if (T.type == 0) {
    int brow = row / T.sub_row_col.x;
    int bcol = col / T.sub_row_col.y;
    local.x = qm_rn_sub(qm_rn_add(qm_rn_add(qm_rn_mul((float)col, px), qm_rn_mul((float)bcol, T.gap.x)), px / 2),
                        T.size.x / 2);
    local.y = T.size.y / 2;
    local.z = qm_rn_sub(qm_rn_add(qm_rn_add(qm_rn_mul((float)row, px), qm_rn_mul((float)brow, T.gap.y)), px / 2),
                        T.size.z / 2);
    local_normal = make_float3(0.f, 1.f, 0.f);
    return false;
  }
  int block = (row / T.sub_row_col.x) * T.row_col.y + col / T.sub_row_col.y;
  const float3 ln = T.local_normals[block];
  const float3 lc = T.local_centers[block];
  row %= T.sub_row_col.x;
  col %= T.sub_row_col.y;
  float3 lp = make_float3(qm_rn_sub(qm_rn_mul(qm_rn_add((float)col, 0.5f), px), T.sub_length.y / 2), 0.0f,
                          qm_rn_sub(qm_rn_mul(qm_rn_add((float)row, 0.5f), px), T.sub_length.x / 2));
  local = qs::add(qs::rotate_to(lp, ln, true), lc);
  local_normal = ln;
  return true;
}

// Frames stored per sub-heliostat (DevGrid::sub_frames): 3 float4 (u, n, v;
// identity flag in u.w).
__device__ __forceinline__ void store_frame(float4* dst, const Frame& f) {
  dst[0] = make_float4(f.u.x, f.u.y, f.u.z, f.identity ? 1.0f : 0.0f);
  dst[1] = make_float4(f.n.x, f.n.y, f.n.z, 0.0f);
  dst[2] = make_float4(f.v.x, f.v.y, f.v.z, 0.0f);
}
__device__ __forceinline__ Frame load_frame(const float4* src) {
  const float4 u = __ldg(src), n = __ldg(src + 1), v = __ldg(src + 2);
  Frame f;
  f.u = make_float3(u.x, u.y, u.z);
  f.n = make_float3(n.x, n.y, n.z);
  f.v = make_float3(v.x, v.y, v.z);
  f.identity = u.w != 0.0f;
  return f;
}

// Both frames of sub-heliostat s of task T for the current sun: the frame
// of its facets' world normal, as facet_geometry + qs::make_frame(normal,
// false) form it, then the flipped frame of its local normal that
// facet_local uses to place focus-flat facets.  Same operations, so the
// tracer's facets are unchanged when it reads them instead.
__device__ __forceinline__ void sub_frames(const DevTask& T, int s, float4* out) {
  Frame hf;
  hf.u = T.fu;
  hf.n = T.fn;
  hf.v = T.fv;
  hf.identity = T.frame_identity != 0;
  const float3 normal = T.type == 1 ? qs::to_world(hf, T.local_normals[s]) : T.normal;
  store_frame(out, qs::make_frame(normal, false));
  if (T.type == 1) store_frame(out + 3, qs::make_frame(T.local_normals[s], true));
  else store_frame(out + 3, qs::make_frame(make_float3(0.f, 1.f, 0.f), true));
}

// Micro-facet at lattice row `row`, column `col` of its heliostat (facet
// id = row * row_col.y * sub_row_col.y + col), in sub-heliostat lattice cell
// (brow, bcol) = (row / sub_row_col.x, col / sub_row_col.y), in world
// space, with the frame of its normal, from its sub-heliostat's stored
// frames (sf: its 6 float4).  The same operations as facet_geometry +
// qs::make_frame (facet_local's lattice arithmetic, its divisions done once
// by the caller), without recomputing the per-sub-heliostat frames.
__device__ __forceinline__ void facet_geometry_framed(const DevTask& T, int row, int col, int brow, int bcol,
                                                      const float4* sf, float3& origin, Frame& normal_frame) {
  Frame hf;
  hf.u = T.fu;
  hf.n = T.fn;
  hf.v = T.fv;
  hf.identity = T.frame_identity != 0;
  const float px = T.pixel_length;
  float3 local;
  if (T.type == 0) {
    local.x = qm_rn_sub(qm_rn_add(qm_rn_add(qm_rn_mul((float)col, px), qm_rn_mul((float)bcol, T.gap.x)), px / 2),
                        T.size.x / 2);
    local.y = T.size.y / 2;
    local.z = qm_rn_sub(qm_rn_add(qm_rn_add(qm_rn_mul((float)row, px), qm_rn_mul((float)brow, T.gap.y)), px / 2),
                        T.size.z / 2);
  } else {
    const int lrow = row - brow * T.sub_row_col.x, lcol = col - bcol * T.sub_row_col.y;
    const float3 lp = make_float3(qm_rn_sub(qm_rn_mul(qm_rn_add((float)lcol, 0.5f), px), T.sub_length.y / 2), 0.0f,
                                  qm_rn_sub(qm_rn_mul(qm_rn_add((float)lrow, 0.5f), px), T.sub_length.x / 2));
    local = qs::add(qs::to_world(load_frame(sf + 3), lp), T.local_centers[brow * T.row_col.y + bcol]);
  }
  origin = qs::add(qs::to_world(hf, local), T.pos);
  normal_frame = load_frame(sf);
}

// Micro-facet f in world space.
__device__ __forceinline__ void facet_geometry(const DevTask& T, int f, float3& origin, float3& normal) {
  Frame hf;
  hf.u = T.fu;
  hf.n = T.fn;
  hf.v = T.fv;
  hf.identity = T.frame_identity != 0;
  float3 local, ln;
  const bool focus_flat = facet_local(T, f, local, ln);
  normal = focus_flat ? qs::to_world(hf, ln) : T.normal;
  origin = qs::add(qs::to_world(hf, local), T.pos);
}

// The task of warp chunk w: the largest t with prefix[t] <= w.  Called by
// all 32 lanes of a warp together: each round the lanes probe 32 points of
// the remaining range at once and a ballot keeps the part holding the
// answer, so the range shrinks 33-fold per round (4 rounds for 87,700 tasks
// instead of 17 dependent halvings).
__device__ __forceinline__ int find_task(const long long* prefix, int n, long long w) {
  const int lane = threadIdx.x & 31;
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const long long span = hi - lo;
    const int probe = lo + (int)(((long long)(lane + 1) * span + 31) / 32);  // in (lo, hi], increasing
    const unsigned below = __ballot_sync(0xffffffffu, __ldg(prefix + probe) <= w);
    const int k = __popc(below);  // probes at or below w: lanes 0 .. k-1 (prefix is nondecreasing)
    const int p_lo = __shfl_sync(0xffffffffu, probe, k > 0 ? k - 1 : 0);
    const int p_hi = __shfl_sync(0xffffffffu, probe, k < 32 ? k : 31);
    if (k > 0) lo = p_lo;
    if (k < 32) hi = p_hi - 1;
  }
  return lo;
}

}  // namespace qm
