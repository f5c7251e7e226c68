// Sun-dependent heliostat geometry, shared by the host scene code and the
// per-sun preparation kernel (csrc/prep.cu), so that a heliostat oriented on
// the GPU is bit-identical to one oriented on the host.
//
// Float work uses the explicitly rounded qs:: operations (plain operators on
// the host, which is built with -ffp-contract=off; _rn intrinsics on the
// device).  The traversal record is built in double with plain operators;
// the device unit that includes this header is compiled with -fmad=false so
// no product is fused there either.
#pragma once

#include "vecmath.h"

namespace qm {

// Heliostat::CSetNormal (Scene/DataStructure/Heliostat/Heliostat.cu:15-20):
// the bisector of the direction to the focus point and the reversed sun
// direction.
QM_HD float3 helio_normal(float3 pos, float3 focus, float3 sun_dir) {
  const float3 reflect_dir = qs::normalize(qs::sub(focus, pos));
  return qs::normalize(qs::sub(reflect_dir, sun_dir));
}

// Heliostat::CSetWorldVertex (Heliostat.cu:22-40): the four corners of the
// mirror plane in world space.
QM_HD void flat_vertices(float3 size, float3 normal, float3 pos, float3 v[4]) {
  v[0] = make_float3(-size.x / 2, size.y / 2, -size.z / 2);
  v[1] = qs::add(make_float3(0, 0, size.z), v[0]);
  v[2] = qs::add(make_float3(size.x, 0, size.z), v[0]);
  v[3] = qs::add(make_float3(size.x, 0, 0), v[0]);
  for (int k = 0; k < 4; ++k) v[k] = qs::add(qs::rotate_to(v[k], normal, false), pos);
}

// Sub-heliostat edge lengths of a focus-flat heliostat: x along z (rows),
// y along x (columns) (FocusFlatRectangleHelio.cu:124-126).
QM_HD float2 sub_lengths(float3 size, float2 gap, int2 row_col) {
  float2 len;
  len.x = qm_rn_div(qm_rn_sub(size.z, qm_rn_mul(gap.y, (float)(row_col.x - 1))), (float)row_col.x);
  len.y = qm_rn_div(qm_rn_sub(size.x, qm_rn_mul(gap.x, (float)(row_col.y - 1))), (float)row_col.y);
  return len;
}

// The three world vertices (B, A, C) of one focus-flat sub-heliostat with
// local centre lc and local normal ln (FocusFlatRectangleHelio.cu:128-131,
// 200-226): each corner of the local parallelogram is turned by the
// sub-heliostat's normal, moved to its centre, turned by the heliostat's
// normal (flipped frame) and moved to the heliostat's position.
QM_HD void focus_flat_sub_vertices(float2 len, float3 lc, float3 ln, float3 normal, float3 pos, float3 out[3]) {
  const float3 local[3] = {make_float3(-len.y / 2, 0.0f, len.x / 2), make_float3(-len.y / 2, 0.0f, -len.x / 2),
                           make_float3(len.y / 2, 0.0f, -len.x / 2)};
  for (int k = 0; k < 3; ++k) {
    float3 p = qs::rotate_to(local[k], ln, true);
    p = qs::add(p, lc);
    p = qs::rotate_to(p, normal, true);
    out[k] = qs::add(p, pos);
  }
}

// Traversal record of one heliostat from its sub-heliostat parallelograms
// (verts: 3 float3 per sub-heliostat, B A C as the reference stores them):
// a padded bounding box in a frame aligned with the sub-heliostat lattice,
// and the lattice itself, so that a ray entering the box only tests the
// sub-heliostats under its path.
//
// Frame: ex along the summed column edges (vertex A -> C of every
// sub-heliostat), ez along the summed row edges (A -> B) made orthogonal to
// ex, and their normal.  Box: the extent of every sub-heliostat corner along
// the three axes, widened by `margin` (1 cm plus 1e-5 of the coordinate
// scale, far above the float rounding of the box and parallelogram tests).
//
// Lattice: column c is assigned the band [x0 + c px, x0 + (c+1) px] along ex,
// row r the band [z0 + r pz, z0 + (r+1) pz] along ez (bands fitted to the
// column and row extents, gap-centred).  The slack is the largest distance by
// which any corner of a sub-heliostat leaves its band; the window margin is
// margin + slack.  A ray hitting sub-heliostat (r, c) does so at a point whose
// ex coordinate lies in column c's band widened by the window margin and
// inside the ray's own ex range within the box, so the columns whose widened
// band meets that range (and likewise the rows) hold every sub-heliostat the
// ray can hit, whatever the geometry: an irregular layout only widens the
// window.  Degenerate frames fall back to a window covering every
// sub-heliostat.
//
// Output (5 float4): centre.xyz + window margin; (ex, half_x); (n, half_n);
// (ez, half_z); (x0, 1/px, z0, 1/pz).  *rows_cols receives the lattice shape.
namespace box_detail {

struct D3 {
  double x, y, z;
};
QM_HD D3 d3(double x, double y, double z) {
  D3 r;
  r.x = x;
  r.y = y;
  r.z = z;
  return r;
}
QM_HD double ddot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
QM_HD D3 dcross(D3 a, D3 b) { return d3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
QM_HD D3 dsub(D3 a, D3 b) { return d3(a.x - b.x, a.y - b.y, a.z - b.z); }
QM_HD bool dunit(D3& a) {
  const double l = sqrt(ddot(a, a));
  if (!(l > 0) || !(l < 1e300)) return false;
  a.x /= l;
  a.y /= l;
  a.z /= l;
  return true;
}
QM_HD double dmin(double a, double b) { return b < a ? b : a; }
QM_HD double dmax(double a, double b) { return a < b ? b : a; }
QM_HD double dabs(double a) { return a < 0 ? -a : a; }

// Corner `corner` (0..3) of sub-heliostat k: A + {0, AB} + {0, AC}.
QM_HD D3 corner(const float3* verts, int k, int corner) {
  const float3 B = verts[3 * k], A = verts[3 * k + 1], C = verts[3 * k + 2];
  const D3 ab = d3((double)B.x - A.x, (double)B.y - A.y, (double)B.z - A.z);
  const D3 ac = d3((double)C.x - A.x, (double)C.y - A.y, (double)C.z - A.z);
  return d3((double)A.x + ((corner & 1) ? ab.x : 0.0) + ((corner & 2) ? ac.x : 0.0),
            (double)A.y + ((corner & 1) ? ab.y : 0.0) + ((corner & 2) ? ac.y : 0.0),
            (double)A.z + ((corner & 1) ? ab.z : 0.0) + ((corner & 2) ? ac.z : 0.0));
}

// Extent along `axis` (relative to `centre`) of lattice column c (by_row
// false) or row c (by_row true).
QM_HD void band_extent(const float3* verts, int rows, int cols, bool by_row, int c, D3 centre, D3 axis, double& lo,
                       double& hi) {
  lo = 1e300;
  hi = -1e300;
  const int n = by_row ? cols : rows;
  for (int j = 0; j < n; ++j) {
    const int k = by_row ? c * cols + j : j * cols + c;
    for (int q = 0; q < 4; ++q) {
      const double x = ddot(dsub(corner(verts, k, q), centre), axis);
      lo = dmin(lo, x);
      hi = dmax(hi, x);
    }
  }
}

// Gap-centred bands of equal pitch fitted to the m column (or row) extents;
// false if the pitch is not positive.  Raises `slack` to the largest
// distance by which an extent leaves its band.
QM_HD bool fit_bands(const float3* verts, int rows, int cols, bool by_row, D3 centre, D3 axis, double& b0,
                     double& pitch, double& slack) {
  const int m = by_row ? rows : cols;
  double gap = 0, l0 = 0, um = 0, prev_hi = 0;
  for (int i = 0; i < m; ++i) {
    double lo, hi;
    band_extent(verts, rows, cols, by_row, i, centre, axis, lo, hi);
    if (i == 0) l0 = lo;
    if (i > 0) gap += lo - prev_hi;
    prev_hi = hi;
    um = hi;
  }
  gap = m > 1 ? gap / (m - 1) : 0.0;
  pitch = (um - l0 + gap) / m;
  b0 = l0 - 0.5 * gap;
  if (!(pitch > 0) || !(pitch < 1e300)) return false;
  for (int i = 0; i < m; ++i) {
    double lo, hi;
    band_extent(verts, rows, cols, by_row, i, centre, axis, lo, hi);
    slack = dmax(slack, (b0 + i * pitch) - lo);
    slack = dmax(slack, hi - (b0 + (i + 1) * pitch));
  }
  return true;
}

}  // namespace box_detail

QM_HD void heliostat_record(const float3* verts, int ns, int2 row_col, float3 pos, float3 normal, float4 out[5],
                            int2* rows_cols) {
  using namespace box_detail;
  int rows = row_col.x, cols = row_col.y;
  bool lattice = ns > 1 && rows > 0 && cols > 0 && rows * cols == ns;
  if (!lattice) {
    rows = 1;
    cols = ns > 1 ? ns : 1;
  }
  D3 ex = d3(0, 0, 0), ez = d3(0, 0, 0), n = d3(0, 0, 0);
  for (int k = 0; k < ns; ++k) {
    const float3 B = verts[3 * k], A = verts[3 * k + 1], C = verts[3 * k + 2];
    ex.x += (double)C.x - A.x;
    ex.y += (double)C.y - A.y;
    ex.z += (double)C.z - A.z;
    ez.x += (double)B.x - A.x;
    ez.y += (double)B.y - A.y;
    ez.z += (double)B.z - A.z;
  }
  bool frame = dunit(ex);
  if (frame) {
    const double p = ddot(ez, ex);
    ez = d3(ez.x - p * ex.x, ez.y - p * ex.y, ez.z - p * ex.z);
    frame = dunit(ez);
  }
  if (frame) {
    n = dcross(ez, ex);
    frame = dunit(n);
  }
  if (!frame) {
    // Any orthonormal frame around the heliostat normal; no lattice.
    n = d3(normal.x, normal.y, normal.z);
    if (!dunit(n)) n = d3(0, 1, 0);
    ex = dabs(n.x) < 0.9 ? d3(0, -n.z, n.y) : d3(-n.y, n.x, 0);
    dunit(ex);
    ez = dcross(ex, n);
    lattice = false;
    rows = 1;
    cols = ns > 1 ? ns : 1;
  }
  const D3 ax[3] = {ex, n, ez};
  const D3 c0 = d3(pos.x, pos.y, pos.z);
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  double maxabs = dabs(c0.x) + dabs(c0.y) + dabs(c0.z);
  for (int k = 0; k < ns; ++k)
    for (int q = 0; q < 4; ++q) {
      const D3 w = corner(verts, k, q);
      const D3 p = dsub(w, c0);
      for (int a = 0; a < 3; ++a) {
        const double d = ddot(p, ax[a]);
        lo[a] = dmin(lo[a], d);
        hi[a] = dmax(hi[a], d);
      }
      maxabs = dmax(maxabs, dabs(w.x) + dabs(w.y) + dabs(w.z));
    }
  const double margin = 0.01 + 1e-5 * maxabs;
  D3 centre = c0;
  double half[3];
  for (int a = 0; a < 3; ++a) {
    const double mid = 0.5 * (lo[a] + hi[a]);
    centre = d3(centre.x + mid * ax[a].x, centre.y + mid * ax[a].y, centre.z + mid * ax[a].z);
    half[a] = 0.5 * (hi[a] - lo[a]) + margin;
  }
  double x0 = 0, px = 1, z0 = 0, pz = 1, slack = 0;
  if (lattice)
    lattice = fit_bands(verts, rows, cols, false, centre, ex, x0, px, slack) &&
              fit_bands(verts, rows, cols, true, centre, ez, z0, pz, slack) && slack < 1e300;
  const double window = lattice ? margin + slack : 1e30;
  if (!lattice) {
    x0 = z0 = 0;
    px = pz = 1;
  }
  out[0] = make_float4((float)centre.x, (float)centre.y, (float)centre.z, (float)window);
  for (int a = 0; a < 3; ++a)
    out[1 + a] = make_float4((float)ax[a].x, (float)ax[a].y, (float)ax[a].z, (float)(half[a] * (1 + 1e-6)));
  // A single column (row) maps every x (z) to band 0.
  out[4] = make_float4((float)x0, cols > 1 ? (float)(1.0 / px) : 0.0f, (float)z0, rows > 1 ? (float)(1.0 / pz) : 0.0f);
  rows_cols->x = rows;
  rows_cols->y = cols;
}

}  // namespace qm
