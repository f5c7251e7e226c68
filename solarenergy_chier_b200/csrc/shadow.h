// Walk-free tests, shared by the host (plain scenes) and the device (batch
// preparation): per heliostat for the shadow walks, per sub-heliostat for
// the block walks.
//
// The reference walks every ray toward the sun through the grid
// (rectGridDDA::collision, rectGridDDA.cu:31-119) and tests the
// sub-heliostats of every heliostat listed in the cells it visits.  A ray of
// heliostat i starts on one of its facets -- inside its padded box, so
// within r_i (the box's half diagonal) of the box centre c -- and travels
// along a sun-shape direction within angle theta of the sun axis a.  Every
// point q of such a ray, at axis parameter s = (q - c).a >= -r_i, lies
// within r_i + (s + r_i) tan(theta) / cos(theta) of the axis line.  So if
// no other heliostat j listed in a cell the rays can visit has its padded
// box within that distance of the axis -- tested as the axis ray against
// box j widened by the distance reached at j's far side, plus a margin far
// above float rounding -- no ray of heliostat i can be shadowed, and its
// shadow walks are skipped with the same result.  The cells a ray can
// visit lie in the grid and inside the same distance of the axis, so they
// are covered by the bounding box of that capsule up to where it leaves the
// grid.  The test is conservative: "false" only means the walks are done.
#pragma once

#include "vecmath.h"

namespace qm {

struct ShadowGrid {
  float3 pos, interval;
  int3 cells;
  const float4* bound;    // 5 float4 per grid-local heliostat (centre, then axes with half extents)
  const int2* ranges;     // [begin, end) of each cell's entries
  const int4* entries;    // grid-local heliostat id first
};

// Ray (o, a) against the box of record b widened by w on every axis: true
// when they meet at an axis parameter >= s_min.
QM_HD bool shadow_box_meets(const float4* b, float w, float3 o, float3 a, float s_min) {
  const float3 r = make_float3(o.x - b[0].x, o.y - b[0].y, o.z - b[0].z);
  float tn = -3.0e38f, tf = 3.0e38f;
  for (int k = 1; k <= 3; ++k) {
    const float4 ax = b[k];
    const float ol = r.x * ax.x + r.y * ax.y + r.z * ax.z;
    const float dl = a.x * ax.x + a.y * ax.y + a.z * ax.z;
    const float half = ax.w + w;
    if (fabsf(dl) < 1e-12f) {
      if (fabsf(ol) > half) return false;
      continue;
    }
    const float t0 = (-half - ol) / dl, t1 = (half - ol) / dl;
    tn = fmaxf(tn, fminf(t0, t1));
    tf = fminf(tf, fmaxf(t0, t1));
  }
  return tn <= tf && tf >= s_min;
}

QM_HD float half_diagonal(const float4* b) { return sqrtf(b[1].w * b[1].w + b[2].w * b[2].w + b[3].w * b[3].w); }

// Rays starting within ri of c, with directions within the angle whose
// tangent is tan_theta of `axis` (not necessarily unit): the heliostats
// other than `own`, listed in a cell the rays can visit, that some of them
// can hit.  Returns their number (each once) and stores the first `cap` of
// them in out[]; -1 when the cone is too wide to enumerate (then any
// heliostat may be hit).  0 means no ray of the cone can hit anything.
QM_HD int cone_candidates(const ShadowGrid& g, int own, float3 c, float ri, float3 axis, float tan_theta, int* out,
                          int cap) {
  if (!(tan_theta >= 0.0f) || tan_theta > 0.5f || !(ri >= 0.0f)) return -1;
  const float al = sqrtf(axis.x * axis.x + axis.y * axis.y + axis.z * axis.z);
  if (!(al > 0.0f)) return -1;
  const float3 a = make_float3(axis.x / al, axis.y / al, axis.z / al);
  const float tq = tan_theta * sqrtf(1.0f + tan_theta * tan_theta) * 1.001f + 1e-6f;
  const float margin = 0.05f + 2e-6f * (fabsf(c.x) + fabsf(c.y) + fabsf(c.z));
  const float3 lo = g.pos;
  const float3 hi = make_float3(g.pos.x + g.cells.x * g.interval.x, g.pos.y + g.cells.y * g.interval.y,
                                g.pos.z + g.cells.z * g.interval.z);
  const float dx = hi.x - lo.x, dy = hi.y - lo.y, dz = hi.z - lo.z;
  // Longest axis run that can matter: inside the grid widened by the widest
  // capsule radius.
  const float s_max = sqrtf(dx * dx + dy * dy + dz * dz) + 4.0f * ri + 10.0f;
  const float R = ri + (s_max + ri) * tq + margin;
  float s_end = s_max;
  {
    // where the axis leaves the grid widened by R
    float tn = -3.0e38f, tf = 3.0e38f;
    const float ov[3] = {c.x, c.y, c.z}, dv[3] = {a.x, a.y, a.z};
    const float lv[3] = {lo.x - R, lo.y - R, lo.z - R}, hv[3] = {hi.x + R, hi.y + R, hi.z + R};
    for (int k = 0; k < 3; ++k) {
      if (fabsf(dv[k]) < 1e-12f) {
        if (ov[k] < lv[k] || ov[k] > hv[k]) return 0;  // the capsule never meets the grid
        continue;
      }
      const float t0 = (lv[k] - ov[k]) / dv[k], t1 = (hv[k] - ov[k]) / dv[k];
      tn = fmaxf(tn, fminf(t0, t1));
      tf = fminf(tf, fmaxf(t0, t1));
    }
    if (tf < -ri) return 0;
    s_end = fminf(s_end, tf);
  }
  const float s0 = -ri;
  const float3 p0 = make_float3(c.x + s0 * a.x, c.y + s0 * a.y, c.z + s0 * a.z);
  const float3 p1 = make_float3(c.x + s_end * a.x, c.y + s_end * a.y, c.z + s_end * a.z);
  const float bmin[3] = {fminf(p0.x, p1.x) - R, fminf(p0.y, p1.y) - R, fminf(p0.z, p1.z) - R};
  const float bmax[3] = {fmaxf(p0.x, p1.x) + R, fmaxf(p0.y, p1.y) + R, fmaxf(p0.z, p1.z) + R};
  const float gp[3] = {lo.x, lo.y, lo.z}, gi[3] = {g.interval.x, g.interval.y, g.interval.z};
  const int gc[3] = {g.cells.x, g.cells.y, g.cells.z};
  int c0[3], c1[3];
  long long count = 1;
  for (int k = 0; k < 3; ++k) {
    const float f0 = floorf((bmin[k] - gp[k]) / gi[k]), f1 = floorf((bmax[k] - gp[k]) / gi[k]);
    if (f1 < 0.0f || f0 > (float)(gc[k] - 1)) return 0;  // no cell of the grid
    c0[k] = f0 < 0.0f ? 0 : (int)f0;
    c1[k] = f1 > (float)(gc[k] - 1) ? gc[k] - 1 : (int)f1;
    count *= (long long)(c1[k] - c0[k] + 1);
  }
  if (count > 8192) return -1;  // too wide to be worth it: walk
  int found = 0;
  for (int x = c0[0]; x <= c1[0]; ++x)
    for (int y = c0[1]; y <= c1[1]; ++y)
      for (int z = c0[2]; z <= c1[2]; ++z) {
        const int cell = (x * gc[1] + y) * gc[2] + z;
        const int2 rg = g.ranges[cell];
        for (int k = rg.x; k < rg.y; ++k) {
          const int j = g.entries[k].x;
          if (j == own) continue;
          bool dup = false;
          for (int q = 0; q < found && q < cap; ++q) dup = dup || out[q] == j;
          if (dup) continue;
          const float4* bj = g.bound + 5 * j;
          const float ex = bj[0].x - c.x, ey = bj[0].y - c.y, ez = bj[0].z - c.z;
          const float D = sqrtf(ex * ex + ey * ey + ez * ez) + half_diagonal(bj);
          const float w = ri + (D + ri) * tq + margin;
          if (!shadow_box_meets(bj, w, c, a, s0 - 1.0f)) continue;
          if (found >= cap) return found + 1;  // more than cap (later ones may repeat: only "> cap" is exact)
          out[found++] = j;
        }
      }
  return found;
}

QM_HD bool cone_free(const ShadowGrid& g, int own, float3 c, float ri, float3 axis, float tan_theta) {
  return cone_candidates(g, own, c, ri, axis, tan_theta, nullptr, 0) == 0;
}

// Shadow walks of heliostat `own`: its rays start on its facets, inside its
// padded box; axis: direction of travel toward the sun; tan_theta: tangent
// of the largest angle between a sun-shape direction and the axis.
QM_HD int shadow_candidates(const ShadowGrid& g, int own, float3 axis, float tan_theta, int* out, int cap) {
  const float4* bi = g.bound + 5 * own;
  return cone_candidates(g, own, make_float3(bi[0].x, bi[0].y, bi[0].z), half_diagonal(bi), axis, tan_theta, out, cap);
}

QM_HD bool shadow_free(const ShadowGrid& g, int own, float3 axis, float tan_theta) {
  return shadow_candidates(g, own, axis, tan_theta, nullptr, 0) == 0;
}

// Block walks of the facets of one sub-heliostat (B, A, C as stored): its
// facets lie on the parallelogram, within half its diagonal of its centre;
// their reflected rays leave within theta_sun + 2 theta_slope of the mirror
// image of the sun's direction of travel about the sub-heliostat's normal
// (reflection keeps angles, and tilting the normal by d turns the reflected
// ray by at most 2 d).  sun: the sun's direction of travel; normal: the
// sub-heliostat's facet normal; theta: theta_sun + 2 theta_slope (radians).
// As cone_candidates: the heliostats that rays of the sub-heliostat's facets
// can hit (-1: too many to enumerate).
QM_HD int block_candidates(const ShadowGrid& g, int own, const float3* bac, float3 sun, float3 normal, float theta,
                           int* out, int cap) {
  if (!(theta >= 0.0f) || theta > 0.45f) return -1;
  const float3 B = bac[0], A = bac[1], C = bac[2];
  const float3 ab = make_float3(B.x - A.x, B.y - A.y, B.z - A.z), ac = make_float3(C.x - A.x, C.y - A.y, C.z - A.z);
  const float3 c = make_float3(A.x + 0.5f * (ab.x + ac.x), A.y + 0.5f * (ab.y + ac.y), A.z + 0.5f * (ab.z + ac.z));
  const float d1 = sqrtf((ab.x + ac.x) * (ab.x + ac.x) + (ab.y + ac.y) * (ab.y + ac.y) + (ab.z + ac.z) * (ab.z + ac.z));
  const float d2 = sqrtf((ab.x - ac.x) * (ab.x - ac.x) + (ab.y - ac.y) * (ab.y - ac.y) + (ab.z - ac.z) * (ab.z - ac.z));
  const float ri = 0.5f * fmaxf(d1, d2) + 0.01f;
  const float sl = sqrtf(sun.x * sun.x + sun.y * sun.y + sun.z * sun.z);
  const float nl = sqrtf(normal.x * normal.x + normal.y * normal.y + normal.z * normal.z);
  if (!(sl > 0.0f) || !(nl > 0.0f)) return -1;
  const float3 s = make_float3(sun.x / sl, sun.y / sl, sun.z / sl), n = make_float3(normal.x / nl, normal.y / nl, normal.z / nl);
  const float k = 2.0f * (s.x * n.x + s.y * n.y + s.z * n.z);
  const float3 axis = make_float3(s.x - k * n.x, s.y - k * n.y, s.z - k * n.z);
  // 1e-4 rad covers the float rounding of the axis and normals
  return cone_candidates(g, own, c, ri, axis, tanf(theta + 1e-4f), out, cap);
}

QM_HD bool block_free(const ShadowGrid& g, int own, const float3* bac, float3 sun, float3 normal, float theta) {
  return block_candidates(g, own, bac, sun, normal, theta, nullptr, 0) == 0;
}

}  // namespace qm
