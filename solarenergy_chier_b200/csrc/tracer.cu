// Quasi-Monte-Carlo heliostat tracer for sm_100a.
//
// One warp owns one micro-facet; its 32 lanes take consecutive light indexes
// (the reference's thread order in map_raytracing, so the 32 rays of a warp
// share an origin and nearly share a direction and their grid walks stay
// together).  A launch covers every facet of every traced heliostat: there
// is no per-heliostat launch, allocation or synchronisation.
//
// Per ray (QuasiMonteCarloRayTracing/RectangleReceiverRectangleGridRayTracing.cu:6-41
// and CylinderReceiverRectangleGridRayTracing.cu:6-40):
//   world-space sun sample, shadow walk toward the sun, slope-error
//   normal, reflection, block walk, receiver hit, energy, flux deposit.
// The walk is the reference's 3D-DDA (QuasiMonteCarloRayTracing/Grid/rectGridDDA.cu:31-119)
// step for step, including its 1e-5 tie rules and truncating start cell.
// Inside a cell each heliostat is first tested against a padded bounding
// box aligned with its sub-heliostat lattice; a ray entering the box tests
// only the sub-heliostats of the lattice rows and columns its path inside
// the box crosses.  Box and window are conservative (padding far above float
// rounding) so the any-hit answer is unchanged.
//
// Everything outside the grid walk (sampling, facet geometry, slope error,
// reflection, receiver intersection, energy) uses explicitly rounded
// operations (qs::), so it rounds exactly as the CPU oracle does.  The grid
// walk and its blocker tests (qm::) are compiled with -fmad=false in the
// exact build (QM_TRACE_VARIANT=exact) and with FMA contraction in the
// production builds.  The approximate-math build (QM_TRACE_APPROX_MATH) also
// evaluates the per-ray arithmetic after the shadow test with FMA
// contraction, the hardware reciprocal square root and approximate
// divisions (qf::); facet geometry stays explicitly rounded.
#include <algorithm>
#include <climits>

#include "device_scene.h"
#include "ray_geom.h"
#include "tracer.h"
#include "vecmath.h"

#ifndef QM_TRACE_VARIANT
#define QM_TRACE_VARIANT fast
#endif
#define QM_CAT2(a, b) a##_##b
#define QM_CAT(a, b) QM_CAT2(a, b)
#define QM_SYM(name) QM_CAT(name, QM_TRACE_VARIANT)

// Per-ray arithmetic outside the walk (slope-error normal, reflection,
// receiver test, energy, pixel index): explicitly rounded (qs::, as the CPU
// oracle rounds it) in every build but the approximate-math one
// (QM_TRACE_APPROX_MATH: qf::, FMA contraction and hardware approximations).
// The receiver-approximate build (QM_TRACE_APPROX_RECEIVER) keeps the
// normal, the reflection and the receiver's decisions explicitly rounded
// and approximates only what follows them: the hit point, (u, v) and the
// energy (cylinder_hit_rx).
#if defined(QM_TRACE_APPROX_MATH)
namespace qx = ::qf;
#define QM_RECEIVER_HIT receiver_hit_approx
#define QM_PIXEL_MUL(a, b) ((a) * (b))
#define QM_ENERGY qf::ray_energy
#elif defined(QM_TRACE_APPROX_RECEIVER)
namespace qx = ::qs;
#define QM_RECEIVER_HIT receiver_hit_rx
#define QM_PIXEL_MUL(a, b) ((a) * (b))
#define QM_ENERGY qf::ray_energy
#else
namespace qx = ::qs;
#define QM_RECEIVER_HIT receiver_hit
#define QM_PIXEL_MUL(a, b) qm_rn_mul((a), (b))
#define QM_ENERGY qs::ray_energy
#endif

namespace qm {
namespace {

// rectGridDDA::absDivide / calTMax / equal / less (rectGridDDA.cuh:15-32).
// The production builds (QM_TRACE_FAST_DIVIDE) divide with the approximate
// reciprocal (within 2 ulp): the quotients only set the order in which the
// walk crosses cell boundaries, which they change only for boundaries within
// a few ulp of a 1e-5 tie.  The exact build divides correctly rounded, as the
// reference does.
__device__ __forceinline__ float abs_divide(float den, float num) {
  if (qm_below_eps(num) && qm_above_neg_eps(num)) return (float)INT_MAX;
#if defined(QM_TRACE_FAST_DIVIDE)
  return fabsf(__fdividef(den, num));
#else
  return fabsf(den / num);
#endif
}
__device__ __forceinline__ float cal_tmax(float dir, float interval, int index, float pos) {
  return fabsf(float(index + (dir >= 0)) * interval - pos);
}
__device__ __forceinline__ bool eq_eps(float a, float b) {
  return ((double)a < (double)b + kEps) && ((double)a > (double)b - kEps);
}
__device__ __forceinline__ bool lt_eps(float a, float b) { return (double)a < (double)b - kEps; }

// Where a - b lies relative to +-1e-5, decided in float when the float
// difference is far enough from both thresholds that its rounding error
// (at most 2^-24 max(|a|,|b|)) cannot change the answer; kUnsure otherwise
// (and for NaN), in which case the caller falls back to the double
// comparisons above.  When it decides, it agrees with them exactly.
enum EpsOrder { kLess = 0, kTied = 1, kGreater = 2, kUnsure = 3 };
__device__ __forceinline__ int eps_order(float a, float b) {
  const float d = a - b;
  const float m = fmaxf(fabsf(a), fabsf(b)) * 1.2e-7f + 1e-30f;
  const float e = 1.0e-5f;
  const float slack = 2.0e-12f;  // covers the float rounding of the 1e-5 constant
  if (d + m < -e - slack) return kLess;
  if (d - m > e + slack) return kGreater;
  if (fabsf(d) + m < e - slack) return kTied;
  return kUnsure;
}

// Conservative slab test along one axis of a heliostat's padded box; ol and
// dl are the ray origin (relative to the box centre) and direction along it.
__device__ __forceinline__ void slab(float ol, float dl, float half, float& tn, float& tf) {
  const float inv = __fdividef(1.0f, dl);
  const float t0 = (-half - ol) * inv;
  const float t1 = (half - ol) * inv;
  tn = fmaxf(tn, fminf(t0, t1));
  tf = fminf(tf, fmaxf(t0, t1));
}

__device__ __forceinline__ int band(float x, float inv_pitch, int n) {
  return (int)fminf(fmaxf(floorf(x * inv_pitch), 0.0f), (float)(n - 1));
}

// The ray against one heliostat's traversal record (5 float4, built by the
// host or the preparation kernel): false if it misses the padded box, else
// the window of lattice rows [r0, r1] and columns [c0, c1] holding every
// sub-heliostat it can hit -- the lattice bands met by the ray's own extent
// inside the box, widened by the record's window margin.  The lattice shape
// (hs: first, count, rows, columns) is read only when the box is entered.
__device__ __forceinline__ bool box_window(const float4* b, const int4* hs, float3 o, float3 d, int& r0, int& r1,
                                           int& c0, int& c1, int& cols) {
  const float4 c = __ldg(b);
  const float3 r = make_float3(o.x - c.x, o.y - c.y, o.z - c.z);
  const float4 an = __ldg(b + 2);
  const float oln = r.x * an.x + r.y * an.y + r.z * an.z;
  const float dln = d.x * an.x + d.y * an.y + d.z * an.z;
  float tn = -3.0e38f, tf = 3.0e38f;
  slab(oln, dln, an.w, tn, tf);
  const float4 ax = __ldg(b + 1);
  const float olx = r.x * ax.x + r.y * ax.y + r.z * ax.z;
  const float dlx = d.x * ax.x + d.y * ax.y + d.z * ax.z;
  slab(olx, dlx, ax.w, tn, tf);
  // Most rays miss here already (the thin plate's slab and one in-plane axis);
  // a third slab can only narrow an empty interval further.
  if (!(tn <= tf && tf >= -1.0f)) return false;
  const float4 az = __ldg(b + 3);
  const float olz = r.x * az.x + r.y * az.y + r.z * az.z;
  const float dlz = d.x * az.x + d.y * az.y + d.z * az.z;
  slab(olz, dlz, az.w, tn, tf);
  if (!(tn <= tf && tf >= -1.0f)) return false;
  tn = fmaxf(tn, -1.0f);
  const int4 lattice = __ldg(hs);  // first, count, rows, columns
  const int rows = lattice.z;
  cols = lattice.w;
  const float4 lat = __ldg(b + 4);  // x0, 1/px, z0, 1/pz
  const float xa = olx + tn * dlx, xb = olx + tf * dlx;
  const float za = olz + tn * dlz, zb = olz + tf * dlz;
  c0 = band(fminf(xa, xb) - c.w - lat.x, lat.y, cols);
  c1 = band(fmaxf(xa, xb) + c.w - lat.x, lat.y, cols);
  r0 = band(fminf(za, zb) - c.w - lat.z, lat.w, rows);
  r1 = band(fmaxf(za, zb) + c.w - lat.z, lat.w, rows);
  return true;
}

// The ray against a heliostat's padded box alone (the test box_window
// opens with): false only if no point of the ray at t >= -1 is inside it.
__device__ __forceinline__ bool box_meets(const float4* b, float3 o, float3 d) {
  const float4 c = __ldg(b);
  const float3 r = make_float3(o.x - c.x, o.y - c.y, o.z - c.z);
  float tn = -3.0e38f, tf = 3.0e38f;
#pragma unroll
  for (int k = 1; k <= 3; ++k) {
    const float4 ax = __ldg(b + k);
    slab(r.x * ax.x + r.y * ax.y + r.z * ax.z, d.x * ax.x + d.y * ax.y + d.z * ax.z, ax.w, tn, tf);
  }
  return tn <= tf && tf >= -1.0f;
}

// Whether the ray hits the parallelogram (a, ab, ac): the reference's test
// (rayParallelogramIntersect, Util/global_function.cuh:101-136), whose
// blocker tests only use the answer.  The exact build divides as the
// reference does.  The production builds compare the numerators against
// |det| instead of dividing by det (u = nu / det lies in [0, 1] exactly when
// nu * sign(det) lies in [0, |det|], and likewise v and t > 1e-5), which
// answers the same except where a rounded quotient lands on a bound.
__device__ __forceinline__ bool parallelogram_hit(float3 orig, float3 dir, float3 a, float3 ab, float3 ac) {
#if defined(QM_TRACE_FAST_DIVIDE)
  const float3 p = cross(dir, ac);
  const float det = dot(ab, p);
  if (qm_below_eps(fabsf(det))) return false;
  const float sg = det > 0.0f ? 1.0f : -1.0f, ad = fabsf(det);
  const float3 tv = sub(orig, a);
  const float nu = dot(tv, p) * sg;
  if (nu < 0.0f || nu > ad) return false;
  const float3 q = cross(tv, ab);
  const float nv = dot(dir, q) * sg;
  if (nv < 0.0f || nv > ad) return false;
  return dot(ac, q) * sg > 1.0e-5f * ad;
#else
  float t, u, v;
  return ray_parallelogram(orig, dir, a, ab, ac, t, u, v);
#endif
}

__device__ __forceinline__ bool sub_hit(const float4* sv, float3 o, float3 d) {
  float4 p0 = __ldg(sv), p1 = __ldg(sv + 1), p2 = __ldg(sv + 2);
  return parallelogram_hit(o, d, make_float3(p0.x, p0.y, p0.z), make_float3(p0.w, p1.x, p1.y),
                           make_float3(p1.z, p1.w, p2.x));
}

// rectGridDDA::intersect over one cell (rectGridDDA.cu:7-25).  A heliostat
// spanning several cells of the walk is listed in each; seen0/seen1 hold the
// last two heliostats this walk tested and missed, whose answer cannot change.
// The reference tests every sub-heliostat of every listed heliostat and
// stops at the first hit; only the answer (hit or not) is used, so testing
// just the sub-heliostats inside the ray's window gives the same answer.
__device__ __forceinline__ bool cell_hit(const DevGrid& g, int cell, int own, float3 o, float3 d, int& seen0,
                                         int& seen1) {
  const int2 range = __ldg(g.cell_range + cell);
  for (int k = range.x; k < range.y; ++k) {
    const int4 en = __ldg(g.entries + k);  // heliostat, first sub-heliostat, count
    const int h = en.x;
    if (h == own || h == seen0 || h == seen1) continue;
    seen1 = seen0;
    seen0 = h;
    if (en.z == 1) {
      if (sub_hit(g.subv + 3 * en.y, o, d)) return true;
      continue;
    }
    int r0, r1, c0, c1, cols;
    if (!box_window(g.bound + 5 * h, g.hsub + h, o, d, r0, r1, c0, c1, cols)) continue;
    for (int rr = r0; rr <= r1; ++rr)
      for (int cc = c0; cc <= c1; ++cc)
        if (sub_hit(g.subv + 3 * (en.y + rr * cols + cc), o, d)) return true;
  }
  return false;
}

// Whether the ray hits any sub-heliostat of heliostat h (the test cell_hit
// makes for each heliostat listed in a cell).
__device__ __forceinline__ bool heliostat_hit(const DevGrid& g, int h, float3 o, float3 d) {
  const int4 hs = __ldg(g.hsub + h);  // first, count, rows, columns
  if (hs.y == 1) return sub_hit(g.subv + 3 * hs.x, o, d);
  int r0, r1, c0, c1, cols;
  if (!box_window(g.bound + 5 * h, g.hsub + h, o, d, r0, r1, c0, c1, cols)) return false;
  for (int rr = r0; rr <= r1; ++rr)
    for (int cc = c0; cc <= c1; ++cc)
      if (sub_hit(g.subv + 3 * (hs.x + rr * cols + cc), o, d)) return true;
  return false;
}

// Any-hit of a ray whose possible blockers are the k listed heliostats
// cand[0..k) (the walk-free tests' candidate lists, 1 <= k): whether the
// reference's walk can find a hit at all.  The production builds
// (QM_TRACE_CANDIDATE_HITS) answer it directly by testing the listed
// heliostats -- the walk visits every cell the ray crosses, so it tests every
// heliostat the ray can hit and finds the same answer, except where a 1e-5
// tie makes it step two axes at once past a cell corner the hit lies in.
// The exact build returns -1 (walk) unless the ray misses every listed
// heliostat's padded box, then 0 (no hit, the walk skipped).
__device__ __forceinline__ int candidate_hit(const DevGrid& g, const int* cand, int k, float3 o, float3 d) {
#if defined(QM_TRACE_CANDIDATE_HITS)
  for (int q = 0; q < k; ++q)
    if (heliostat_hit(g, __ldg(cand + q), o, d)) return 1;
  return 0;
#else
  for (int q = 0; q < k; ++q)
    if (box_meets(g.bound + 5 * __ldg(cand + q), o, d)) return -1;
  return 0;
#endif
}

// rectGridDDA::collision (rectGridDDA.cu:31-119).  The reference loops until
// the walk leaves the grid; a walk that stops advancing (an exact tie the
// reference never leaves) or exceeds cells.x+cells.y+cells.z+2 steps ends
// here with "no hit" and a diagnostic count instead.
// Start of a walk from origin o: its cell, and per axis the distances to the
// cell's lower and upper boundary (rectGridDDA.cu:36-52; calTMax with
// dir < 0 and dir >= 0).  It depends on the origin only.
struct WalkStart {
  int3 cell;
  float3 lo, hi;
};
__device__ __forceinline__ WalkStart walk_start(const DevGrid& g, float3 o) {
  WalkStart w;
  const float3 rel = make_float3(o.x - g.pos.x, o.y - g.pos.y, o.z - g.pos.z);
  w.cell = trunc3(cdiv(rel, g.interval));
  w.lo = make_float3(cal_tmax(-1.0f, g.interval.x, w.cell.x, rel.x), cal_tmax(-1.0f, g.interval.y, w.cell.y, rel.y),
                     cal_tmax(-1.0f, g.interval.z, w.cell.z, rel.z));
  w.hi = make_float3(cal_tmax(1.0f, g.interval.x, w.cell.x, rel.x), cal_tmax(1.0f, g.interval.y, w.cell.y, rel.y),
                     cal_tmax(1.0f, g.interval.z, w.cell.z, rel.z));
  return w;
}

__device__ __forceinline__ bool collide(const DevGrid& g, int own, float3 o, float3 d, const WalkStart& w,
                                        unsigned& flags) {
  int3 c = w.cell;
  int3 st = make_int3(d.x >= 0 ? 1 : -1, d.y >= 0 ? 1 : -1, d.z >= 0 ? 1 : -1);
  float3 tm, td;
  tm.x = abs_divide(d.x >= 0 ? w.hi.x : w.lo.x, d.x);
  tm.y = abs_divide(d.y >= 0 ? w.hi.y : w.lo.y, d.y);
  tm.z = abs_divide(d.z >= 0 ? w.hi.z : w.lo.z, d.z);
  td.x = abs_divide(g.interval.x, d.x);
  td.y = abs_divide(g.interval.y, d.y);
  td.z = abs_divide(g.interval.z, d.z);
  int seen0 = -1, seen1 = -1;
  for (int it = 0; it < g.max_steps; ++it) {
    if ((unsigned)c.x >= (unsigned)g.cells.x || (unsigned)c.y >= (unsigned)g.cells.y ||
        (unsigned)c.z >= (unsigned)g.cells.z)
      return false;
    int cell = c.x * g.cells.y * g.cells.z + c.y * g.cells.z + c.z;
    if (cell_hit(g, cell, own, o, d, seen0, seen1)) return true;
    bool sx = false, sy = false, sz = false;
    // Common case: one boundary is nearer than both others by more than
    // 1e-5 plus the float rounding of the difference (tm >= 0, so the error
    // of tm_j - min is at most 2^-24 tm_j).  The reference's rules then step
    // that axis alone, whatever the order of the other two.
    const float mn = fminf(fminf(tm.x, tm.y), tm.z);
    const float c0 = 1.0e-5f + 2.0e-12f;
    const bool gx = tm.x - mn > fmaf(tm.x, 1.2e-7f, c0);
    const bool gy = tm.y - mn > fmaf(tm.y, 1.2e-7f, c0);
    const bool gz = tm.z - mn > fmaf(tm.z, 1.2e-7f, c0);
    if ((int)gx + (int)gy + (int)gz == 2) {
      if (!gx) { c.x += st.x; tm.x += td.x; }
      else if (!gy) { c.y += st.y; tm.y += td.y; }
      else { c.z += st.z; tm.z += td.z; }
      continue;
    }
    const int xy = eps_order(tm.x, tm.y);
    const int xz = eps_order(tm.x, tm.z);
    const int yz = eps_order(tm.y, tm.z);
    if (xy != kUnsure && xz != kUnsure && yz != kUnsure) {
      // less(a,b) <=> kLess, equal(a,b) <=> kTied, less(b,a) <=> kGreater
      if (xy == kLess) {
        if (xz != kGreater) { c.x += st.x; sx = true; }
        if (xz != kLess) { c.z += st.z; sz = true; }
      } else if (xy == kGreater) {
        if (yz != kGreater) { c.y += st.y; sy = true; }
        if (yz != kLess) { c.z += st.z; sz = true; }
      } else {
        if (xz != kGreater) { c.x += st.x; c.y += st.y; sx = sy = true; }
        if (xz != kLess) { c.z += st.z; sz = true; }
      }
    } else if (lt_eps(tm.x, tm.y)) {
      if (lt_eps(tm.x, tm.z) || eq_eps(tm.x, tm.z)) { c.x += st.x; sx = true; }
      if (lt_eps(tm.z, tm.x) || eq_eps(tm.x, tm.z)) { c.z += st.z; sz = true; }
    } else if (lt_eps(tm.y, tm.x)) {
      if (lt_eps(tm.y, tm.z) || eq_eps(tm.y, tm.z)) { c.y += st.y; sy = true; }
      if (lt_eps(tm.z, tm.y) || eq_eps(tm.y, tm.z)) { c.z += st.z; sz = true; }
    } else {
      if (lt_eps(tm.x, tm.z) || eq_eps(tm.x, tm.z)) { c.x += st.x; c.y += st.y; sx = sy = true; }
      if (lt_eps(tm.z, tm.x) || eq_eps(tm.x, tm.z)) { c.z += st.z; sz = true; }
    }
    if (!(sx || sy || sz)) {
      flags |= 2u;
      return false;
    }
    tm.x += sx ? td.x : 0;
    tm.y += sy ? td.y : 0;
    tm.z += sz ? td.z : 0;
  }
  flags |= 2u;
  return false;
}

// Rays of one launch: for task t (a heliostat), rays r in [0, F_t * nl) with
// facet f = r / nl and light l = light_begin + r % nl, nl = lights per facet.
// Each warp takes one chunk of kChunk consecutive rays of one task (task ray
// counts are padded to whole chunks, so a chunk never straddles heliostats);
// lane i handles rays i, i+32, i+64, ... of the chunk.  With nl >= 32 the 32
// rays of an iteration share a facet; with fewer lights per facet several
// facets share a warp and no lane idles.
//
// Facet window: the facets of an iteration lie within 32 consecutive ids
// (at most ceil(32/nl) + 1 <= 32 of them), so a warp keeps a window of 32
// facets in shared memory -- origin, normal frame and the two pool offsets --
// computed one facet per lane, and refills it only when an iteration needs a
// facet past its end (once per 32 facets: twice per chunk of 2,048 rays at
// 32 lights per facet).  Per-ray work then reads
// the window instead of re-deriving the facet, and holds no facet state in
// registers across the grid walks.
#ifndef QM_TRACE_THREADS
#define QM_TRACE_THREADS 256
#endif
constexpr int kThreads = QM_TRACE_THREADS;
constexpr int kWindow = 32;

struct FacetWindow {
  // Per warp: the task's sample pools (P + L entries each, so an offset
  // g in [0, P) plus a light index in [0, L) needs no wrap-around).
  const float4* samples[kThreads / 32];
  const float4* perturbations[kThreads / 32];
  int shadow_free[kThreads / 32];  // the task's shadow-walk code (DevTask::shadow_free)
  float4 o[kThreads];   // origin.xyz, pool offset g[f] (int bits)
  float4 u[kThreads];   // frame u.xyz, pool offset g[(f+1) % P] (int bits; bit 31: block walk skippable)
  float4 n[kThreads];   // frame n.xyz, sub-heliostat << 4 | candidate blockers << 1 | frame identity (int bits)
  float4 v[kThreads];   // frame v.xyz
};

// Shared-memory read the compiler may not merge with an earlier read of the
// same slot: facet data is re-read where it is used instead of being held in
// registers across a grid walk.
__device__ __forceinline__ float4 lds(const float4& x) {
  float4 r;
  const unsigned a = (unsigned)__cvta_generic_to_shared(&x);
  asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(r.x), "=f"(r.y), "=f"(r.z), "=f"(r.w) : "r"(a));
  return r;
}

__device__ __forceinline__ int lds_int(const int& x) {
  int r;
  const unsigned a = (unsigned)__cvta_generic_to_shared(&x);
  asm volatile("ld.shared.s32 %0, [%1];" : "=r"(r) : "r"(a));
  return r;
}

__device__ __forceinline__ const float4* lds_ptr(const float4* const& x) {
  unsigned long long r;
  const unsigned a = (unsigned)__cvta_generic_to_shared(&x);
  asm volatile("ld.shared.u64 %0, [%1];" : "=l"(r) : "r"(a));
  return reinterpret_cast<const float4*>(r);
}

// DDA start of a facet's walks, computed from its origin when a ray walks
// (most rays decide shadowing and blocking without a walk).
__device__ __forceinline__ WalkStart window_start(const DevGrid& g, const FacetWindow& win, int slot) {
  return walk_start(g, xyz(lds(win.o[slot])));
}

// Output of a launch: flux into the receiver images (nearest pixel, the
// reference's deposit), per-ray outcome codes, or the differentiable
// forward's bilinear deposit plus one hit bit per ray.
// Outputs: flux image (plain path), per-ray outcome codes, bilinear FP64
// deposit + hit bits (differentiable forward), hit bits alone (the adjoint
// recomputing its hit records).
enum TraceOut { kOutFlux = 0, kOutRecord = 1, kOutSplat = 2, kOutBits = 3 };

// Bilinear deposit of energy e at continuous pixel position (X, Y) (pixel c
// spans [c, c+1), centres at c + 0.5): columns wrap around for a cylinder
// (its columns are angles), everything else outside the image is dropped.
// Accumulated in FP64, so the deposit (and the loss computed from it) does
// not depend on the order of the atomic additions.
__device__ __forceinline__ void splat_bilinear(const DevReceiver& R, float X, float Y, float e) {
  const float x = X - 0.5f, y = Y - 0.5f;
  const float x0 = floorf(x), y0 = floorf(y);
  const float fx = x - x0, fy = y - y0;
  const int c0 = (int)x0, r0 = (int)y0;
  const int w = R.resolution.x, h = R.resolution.y;
  const bool wrap = R.type == 1;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    int c = c0 + (k & 1), r = r0 + (k >> 1);
    const float wgt = ((k & 1) ? fx : 1.0f - fx) * ((k >> 1) ? fy : 1.0f - fy);
    if (wrap) c = c < 0 ? c + w : (c >= w ? c - w : c);
    if (c < 0 || c >= w || r < 0 || r >= h) continue;
    atomicAdd(R.deposit + r * w + c, (double)(e * wgt));
  }
}

// The persistent build's kernels take the launch's work counter as a second
// argument; the other builds keep TraceParams as their only argument.
#if defined(QM_TRACE_PERSISTENT)
#define QM_TRACE_ARGS TraceParams p, unsigned long long* work_counter
#else
#define QM_TRACE_ARGS TraceParams p
#endif

template <int kOut>
#ifndef QM_TRACE_MIN_BLOCKS
#define QM_TRACE_MIN_BLOCKS 4
#endif
__global__ void __launch_bounds__(kThreads, QM_TRACE_MIN_BLOCKS) trace_kernel(QM_TRACE_ARGS) {
  __shared__ FacetWindow win;
  const int lane = threadIdx.x & 31;
  const int wbase = threadIdx.x & ~31;  // this warp's 32 window slots
#if defined(QM_TRACE_PERSISTENT)
  long long warp = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
#else
  const long long warp = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
#endif
  const int nl = p.light_end - p.light_begin;
#if defined(QM_TRACE_PERSISTENT)
  // Persistent flux launches: a grid of resident warps, each taking the next
  // warp chunk from the launch's work counter (zeroed by the launcher) until
  // none is left; `warp` is then the chunk's index within the launch.  Other
  // outputs keep one warp per chunk.
  const bool persistent = kOut == kOutFlux && work_counter;
  for (;;) {
    if (persistent) {
      long long w = 0;
      if (lane == 0) w = (long long)atomicAdd(work_counter, 1ull);
      warp = __shfl_sync(0xffffffffu, w, 0);
      if (warp >= p.total_facets - p.chunk_begin) return;
      __syncwarp();
    }
#endif
  // Ray indexes within one heliostat fit in int: the host refuses launches
  // with num_facets * lights >= 2^31.
  int t, r0, r_end;
  if (kOut == kOutRecord) {
    const long long span = (long long)(p.record_facet_end - p.record_facet_begin) * nl;
    if (warp * kChunk >= span) return;
    t = p.record_task;
    r0 = p.record_facet_begin * nl + (int)warp * kChunk;
    r_end = p.record_facet_end * nl;
  } else {
    const long long chunk = p.chunk_begin + warp;
    if (chunk >= p.total_facets) return;  // total_facets holds the end chunk
    t = find_task(p.facet_prefix, p.num_tasks, chunk);
    r0 = (int)(chunk - __ldg(p.facet_prefix + t)) * kChunk;
    r_end = p.tasks[t].num_facets * nl;
  }
  // The task stays in global memory (L1-resident) and is read where used.
  const DevTask& T = p.tasks[t];
  const DevGrid& G = p.grids[T.grid];
  const DevReceiver& R = p.receivers[T.receiver];
  if (lane == 0) {
    win.shadow_free[threadIdx.x >> 5] = T.shadow_free;
    win.samples[threadIdx.x >> 5] = T.samples;
    win.perturbations[threadIdx.x >> 5] = T.perturbations;
  }
  __syncwarp();
  // This lane's first ray; later rays advance by 32 = q32 * nl + r32.
  int f = (r0 + lane) / nl;
  int l = (r0 + lane) - f * nl;
  const int q32 = p.lights_q32, r32 = p.lights_r32;
  const int iters = min(kChunkIters, (r_end - r0 + 31) >> 5);  // warp-uniform

  unsigned flags = 0;
  double power = 0.0;
  unsigned long long clamped = 0;
  int base = 0;        // first facet id of the window
  bool filled = false;  // warp-uniform
  for (int it = 0; it < iters; ++it) {
    const bool active = r0 + it * 32 + lane < r_end;
    bool hit = false;
    // Lane 0 holds the smallest facet of the iteration (it is active whenever
    // any lane is) and every facet of the iteration lies within 31 of it.
    const int f0 = __shfl_sync(0xffffffffu, f, 0);
    if (__any_sync(0xffffffffu, active && (!filled || f - base >= kWindow))) {
      __syncwarp();
      base = f0;
      filled = true;
      const int fw = base + lane;
      if (fw < T.num_facets) {
        // Lattice position of the facet: row, column, and its sub-heliostat
        // lattice cell (flat heliostats have one sub-heliostat).
        const int per_row = T.row_col.y * T.sub_row_col.y;
        const int frow = fw / per_row, fcol = fw - frow * per_row;
        const int brow = frow / T.sub_row_col.x, bcol = fcol / T.sub_row_col.y;
        const int block = T.type == 1 ? brow * T.row_col.y + bcol : 0;
        const int sub = __ldg(&G.hsub[T.own].x) + block;
        // The facet and the frame of its normal, from its sub-heliostat's
        // frames (computed once per sun with the walk codes).
        float3 origin;
        Frame fr;
        facet_geometry_framed(T, frow, fcol, brow, bcol, G.sub_frames + 6 * sub, origin, fr);
        win.o[wbase + lane] = make_float4(origin.x, origin.y, origin.z, __int_as_float(__ldg(T.offsets + fw)));
        // Pool offsets lie below 2^30; bit 31 carries the facet's
        // sub-heliostat block-free flag, and the frame word below its
        // candidate blockers (qm::block_candidates): n.w = sub-heliostat << 4
        // | candidates << 1 | frame identity.
        const int bcode = __ldg(G.sub_free + sub);
        const int free_bit = bcode == 1 ? (int)0x80000000 : 0;
        const int cands = bcode >= 2 ? bcode - 1 : 0;
        win.u[wbase + lane] = make_float4(fr.u.x, fr.u.y, fr.u.z,
                                          __int_as_float(__ldg(T.offsets + (fw + 1) % T.pool_size) | free_bit));
        win.n[wbase + lane] = make_float4(fr.n.x, fr.n.y, fr.n.z, __int_as_float((sub << 4) | (cands << 1) | (fr.identity ? 1 : 0)));
        win.v[wbase + lane] = make_float4(fr.v.x, fr.v.y, fr.v.z, 0.0f);
      }
      __syncwarp();
    }
    if (active) {
      const int slot = wbase + (f - base);
      const int lab = p.light_begin + l;
      // Pool offsets lie in [0, P) and light indexes in [0, L); the pools hold
      // P + L entries (entry P + i repeats entry i), so (g + l) % P needs no
      // modulo.  The sun-shape pool is stored already turned by the sun
      // frame (world space).
      const float3 dir = xyz(__ldg(lds_ptr(win.samples[threadIdx.x >> 5]) + __float_as_int(win.o[slot].w) + lab));
      int32_t code;
      // Heliostats whose rays no other heliostat can shadow skip the shadow
      // walk; where only a few listed heliostats can (qm::cone_candidates,
      // decided per sun when the task is built), candidate_hit decides.
      const int sc = lds_int(win.shadow_free[threadIdx.x >> 5]);
      int shadowed = sc == 1 ? 0 : -1;  // -1: walk
      if (sc >= 2) shadowed = candidate_hit(G, T.shadow_cand, sc - 1, xyz(lds(win.o[slot])), dir);
      if (shadowed < 0) shadowed = collide(G, T.own, xyz(lds(win.o[slot])), dir, window_start(G, win, slot), flags);
      if (shadowed) {
        code = kShadowed;
      } else {
        Frame nframe;
        nframe.u = xyz(win.u[slot]);
        const float4 wn = win.n[slot];
        nframe.n = xyz(wn);
        nframe.v = xyz(win.v[slot]);
        nframe.identity = (__float_as_int(wn.w) & 1) != 0;
        const int g1 = __float_as_int(lds(win.u[slot]).w);
        const int b = (g1 & 0x7fffffff) + lab;
        // Both normalisations take vectors of unit scale: the pools hold unit
        // vectors (qmcrt_set_sample_pool refuses squared lengths outside
        // [0.25, 4]), the facet frames are orthonormal (or NaN), and the
        // reflection keeps the direction's length, so the squared lengths lie
        // far inside the series' range [2^-125, 2^125) and normalize_unit
        // drops the range test.
        float3 n = qx::normalize_unit(qx::to_world(nframe, xyz(__ldg(lds_ptr(win.perturbations[threadIdx.x >> 5]) + b))));
        float3 rd = qx::normalize_unit(qx::reflect(neg(dir), n));
        // Facets of sub-heliostats no other heliostat can block skip the
        // block walk; where only a few listed heliostats can
        // (qm::block_candidates, decided per sun with the pools),
        // candidate_hit decides.
        int blocked = 0;
        if (g1 >= 0) {
          const int nw = __float_as_int(lds(win.n[slot]).w);
          const int k = (nw >> 1) & 7;
          blocked = k ? candidate_hit(G, G.sub_cand + kMaxCandidates * (nw >> 4), k, xyz(lds(win.o[slot])), rd) : -1;
          if (blocked < 0) blocked = collide(G, T.own, xyz(lds(win.o[slot])), rd, window_start(G, win, slot), flags);
        }
        if (blocked) {
          code = kBlocked;
        } else {
          float tt, uu, vv;
          if (!QM_RECEIVER_HIT(R, xyz(lds(win.o[slot])), rd, tt, uu, vv)) {
            code = kMissed;
          } else {
            float e = QM_ENERGY(tt, rd, n, T.factor);
            if (kOut == kOutBits) {
              code = 0;
            } else if (kOut == kOutSplat) {
              splat_bilinear(R, QM_PIXEL_MUL(vv, (float)R.resolution.x), QM_PIXEL_MUL(uu, (float)R.resolution.y), e);
              power += (double)e;
              code = 0;
            } else {
            int row = int(QM_PIXEL_MUL(uu, (float)R.resolution.y));
            int col = int(QM_PIXEL_MUL(vv, (float)R.resolution.x));
            if (row >= R.resolution.y || col >= R.resolution.x || row < 0 || col < 0) {
              row = min(max(row, 0), R.resolution.y - 1);
              col = min(max(col, 0), R.resolution.x - 1);
              ++clamped;
            }
            const int pix = row * R.resolution.x + col;
            atomicAdd(R.image + pix, e);
            power += (double)e;
            code = pix;
            }
          }
        }
      }
      if (kOut == kOutRecord) p.records[(size_t)(f - p.record_facet_begin) * nl + l] = code;
      if (kOut == kOutSplat || kOut == kOutBits) hit = code >= 0;
    }
    if (kOut == kOutSplat || kOut == kOutBits) {
      const unsigned bits = __ballot_sync(0xffffffffu, hit);
      if (lane == 0 && p.hit_bits) p.hit_bits[warp * kChunkIters + it] = bits;
    }
    f += q32;
    l += r32;
    if (l >= nl) {
      l -= nl;
      ++f;
    }
  }
  for (int off = 16; off > 0; off >>= 1) {
    power += __shfl_down_sync(0xffffffffu, power, off);
    clamped += __shfl_down_sync(0xffffffffu, clamped, off);
  }
  flags = __reduce_or_sync(0xffffffffu, flags);
  if (lane == 0) {
    if (p.chunk_power && kOut != kOutRecord) p.chunk_power[warp] = power;
    else if (power != 0.0) atomicAdd(p.power + T.power_slot, power);
    if (clamped) atomicAdd(p.diag + kDiagClamped, clamped);
    if (flags & 2u) atomicAdd(p.diag + kDiagDdaCap, 1ull);
  }
#if defined(QM_TRACE_PERSISTENT)
    if (!persistent) return;
  }
#endif
}

__global__ void facets_kernel(DevTask T, float3* origins, float3* normals) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= T.num_facets) return;
  float3 o, n;
  facet_geometry(T, f, o, n);
  origins[f] = o;
  normals[f] = n;
}

}  // namespace

cudaError_t QM_SYM(launch_facets)(const DevTask& task, float3* origins, float3* normals, cudaStream_t stream) {
  if (task.num_facets <= 0) return cudaSuccess;
  const int threads = 256;
  facets_kernel<<<(task.num_facets + threads - 1) / threads, threads, 0, stream>>>(task, origins, normals);
  return cudaGetLastError();
}

int QM_SYM(trace_chunk_rays)() { return kChunk; }

cudaError_t QM_SYM(launch_trace)(const TraceParams& params, int out, cudaStream_t stream,
                                 unsigned long long* work_counter) {
  const int threads = kThreads;
  const long long nl = params.light_end - params.light_begin;
  if (nl <= 0) return cudaSuccess;
  TraceParams p = params;
  p.lights_q32 = (int)(32 / nl);
  p.lights_r32 = (int)(32 % nl);
  const bool record = out == kOutRecord;
  const long long warps = record ? ((long long)(p.record_facet_end - p.record_facet_begin) * nl + kChunk - 1) / kChunk
                                 : p.total_facets - p.chunk_begin;
  if (!record && p.chunk_begin < 0) return cudaErrorInvalidValue;
  if (warps <= 0) return cudaSuccess;
  long long blocks = (warps + (threads / 32) - 1) / (threads / 32);
  if (blocks > 0x7fffffffLL) return cudaErrorInvalidValue;
#if defined(QM_TRACE_PERSISTENT)
  if (out == kOutFlux && work_counter) {
    // as many blocks as stay resident together, never more than the chunks
    static int resident = 0;
    if (!resident) {
      int dev = 0, sms = 0, per_sm = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trace_kernel<kOutFlux>, threads, 0);
      resident = std::max(1, sms * per_sm);
    }
    blocks = std::min<long long>(blocks, resident);
    cudaError_t e = cudaMemsetAsync(work_counter, 0, sizeof(unsigned long long), stream);
    if (e != cudaSuccess) return e;
  } else {
    work_counter = nullptr;
  }
#define QM_TRACE_LAUNCH_ARGS p, work_counter
#else
  (void)work_counter;
#define QM_TRACE_LAUNCH_ARGS p
#endif
  switch (out) {
    case kOutRecord: trace_kernel<kOutRecord><<<(unsigned)blocks, threads, 0, stream>>>(QM_TRACE_LAUNCH_ARGS); break;
    case kOutSplat: trace_kernel<kOutSplat><<<(unsigned)blocks, threads, 0, stream>>>(QM_TRACE_LAUNCH_ARGS); break;
    case kOutBits: trace_kernel<kOutBits><<<(unsigned)blocks, threads, 0, stream>>>(QM_TRACE_LAUNCH_ARGS); break;
    default: trace_kernel<kOutFlux><<<(unsigned)blocks, threads, 0, stream>>>(QM_TRACE_LAUNCH_ARGS); break;
  }
  return cudaGetLastError();
}

}  // namespace qm
