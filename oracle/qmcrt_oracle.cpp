// CPU ORACLE - test infrastructure only.
//
// A CPU restatement of SolarEnergy_Chier's QuasiMonteCarloRayTracer path,
// used by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg as
// the checker.  Nothing in the product (solarenergy_chier_b200/) links,
// loads or calls this file.
//
// C++17, compiled by g++ with -O2 -ffp-contract=off -fopenmp and no CUDA.
// Every routine is templated on the arithmetic type:
//   float  - the per-ray parity oracle: the reference's float operations in
//            the reference's order, IEEE rounding, 1/sqrtf for rsqrtf (the
//            reference's host definition, Util/vector_arithmetic.cuh:51-54),
//            comparisons with the 1e-5 tolerance done in double as the
//            reference's double literal makes them;
//   double - the accuracy oracle: the same algorithm in double precision.
// Each function cites the reference file:line it restates.  Parity pins:
// tests/test_oracle_golden.py checks this file against the known answers of
// the reference's own gtest suites, and tests/golden/ holds outputs of the
// reference's own code (see tests/golden/make_golden.py).
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace oracle {

constexpr double EPS = 1e-5;  // Util/global_constant.h:11

template <class T>
struct V {
  T x, y, z;
};
template <class T> V<T> mk(T x, T y, T z) { return V<T>{x, y, z}; }
template <class T> V<T> operator+(V<T> a, V<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> V<T> operator-(V<T> a, V<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> V<T> operator-(V<T> a) { return {-a.x, -a.y, -a.z}; }
template <class T> V<T> operator*(V<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> V<T> plus_s(V<T> a, T s) { return {a.x + s, a.y + s, a.z + s}; }
template <class T> V<T> minus_s(V<T> a, T s) { return {a.x - s, a.y - s, a.z - s}; }
template <class T> V<T> cwise_div(V<T> a, V<T> b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
template <class T> T dot(V<T> a, V<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> V<T> cross(V<T> a, V<T> b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// Reciprocal square root used by normalize: correctly rounded.  In float it
// is 1/sqrt evaluated in double and rounded once, which is what the
// reference's nvcc host build computes for rsqrtf (established output for
// output on 1.2e8 inputs; the reference's own non-nvcc fallback
// 1.0f/sqrtf(x), Util/vector_arithmetic.cuh:51-54, rounds twice and differs
// in about a third of cases).
inline float inv_sqrt(float x) { return (float)(1.0 / std::sqrt((double)x)); }
inline double inv_sqrt(double x) { return 1.0 / std::sqrt(x); }
template <class T> V<T> normalize(V<T> v) { T s = inv_sqrt(dot(v, v)); return v * s; }
template <class T> T length(V<T> v) { return std::sqrt(dot(v, v)); }
template <class T> V<T> reflect(V<T> i, V<T> n) { return i - (n * T(2)) * dot(n, i); }
template <class T> V<T> half_of(V<T> v) { T inv = T(1) / T(2); return v * inv; }

template <class T, class U> V<T> cast(V<U> v) { return {T(v.x), T(v.y), T(v.z)}; }

// global_func::local2world_rotate (Util/global_function.cuh:19-36) and the
// focus-flat variant (FocusFlatRectangleHelio.cuh:16-46, flip = true).
template <class T>
V<T> rotate(V<T> d, V<T> n, bool flip) {
  if ((double)std::fabs(n.x) < EPS && (double)std::fabs(n.z) < EPS) return d;
  V<T> u = normalize(cross(mk<T>(0, 1, 0), n));
  V<T> v = normalize(cross(u, n));
  if (flip && n.z < 0) {
    u = -u;
    v = -v;
  }
  return mk<T>(d.x * u.x + d.y * n.x + d.z * v.x, d.x * u.y + d.y * n.y + d.z * v.y,
               d.x * u.z + d.y * n.z + d.z * v.z);
}

// global_func::rotateY (Util/global_function.cuh:51-59).
template <class T>
V<T> rotate_yaw(V<T> p, V<T> from, V<T> to) {
  int s = (cross(from, to).y > 0) ? 1 : -1;
  T c = dot(from, to);
  T sn = T(s) * std::sqrt(T(1) - c * c);
  return mk<T>(c * p.x + sn * p.z, p.y, -sn * p.x + c * p.z);
}

// global_func::rayParallelogramIntersect (Util/global_function.cuh:101-136),
// stage counters for the algorithmic-work census.
struct Census {
  long long tests_det = 0, tests_u = 0, tests_v = 0, tests_t = 0, cells = 0;
};

template <class T>
bool parallelogram(V<T> o, V<T> d, V<T> A, V<T> B, V<T> C, T& t, T& u, T& v, Census* cz) {
  V<T> ab = B - A, ac = C - A;
  V<T> p = cross(d, ac);
  T det = dot(ab, p);
  if (cz) ++cz->tests_det;
  if ((double)std::fabs(det) < EPS) return false;
  V<T> tv = o - A;
  if (cz) ++cz->tests_u;
  u = dot(tv, p) / det;
  if (u < 0 || u > 1) return false;
  V<T> q = cross(tv, ab);
  if (cz) ++cz->tests_v;
  v = dot(d, q) / det;
  if (v < 0 || v > 1) return false;
  if (cz) ++cz->tests_t;
  t = dot(ac, q) / det;
  if ((double)t < EPS) return false;
  return true;
}

// ---------------------------------------------------------------------------
// Scene description, as parsed from the .scn / .json files (float inputs).
struct Desc {
  float sun_dir[3];
  float dni, csr, recv_px, helio_px, rho, sigma;
  int groups, per_group, its_groups;
  int n_recv;
  const int* recv_type;
  const float* recv_pos;
  const float* recv_size;
  const float* recv_norm;
  const int* recv_face;
  int n_grid;
  const int* grid_type;
  const float* grid_pos;
  const float* grid_size;
  const float* grid_inter;
  const int* grid_n;
  const int* grid_htype;
  const int* grid_start;
  const int* grid_recv;
  int n_helio;
  const int* h_type;
  const float* h_pos;
  const float* h_size;
  const float* h_gap;
  const int* h_matrix;
  const float* h_surface;  // 6 per heliostat
  const int* h_grid;
  const int* h_local_off;  // index of first file centre (or -1)
  const float* local_centers;
  const float* local_normals;
};

template <class T>
struct Recv {
  int type, face;
  V<T> pos, size, normal, local_normal, vert[4], focus;
  T pixel_length;
  int res_x, res_y;
};

template <class T>
struct Helio {
  int type, grid, n_sub, sub_begin, n_facets, read_method;
  V<T> pos, size, normal, vertex[4];
  T gap_x, gap_y, focus_length, pixel_length;
  int rows, cols, sub_rows, sub_cols;
  T len_x, len_y;  // sub-heliostat length along z (rows) and along x (columns)
  std::vector<V<T>> lc, ln;  // focus-flat local centres / normals
  std::vector<V<T>> file_c, file_n;
};

template <class T>
struct Grid {
  V<T> pos, size, inter;
  int nx, ny, nz, start, count, recv;
  std::vector<int> index, match;  // reference CSR (sub-heliostat ids)
  std::vector<V<T>> verts;        // 3 per sub-heliostat
};

template <class T>
struct Scene {
  V<T> sun;
  T dni, rho;
  int per_group;
  std::vector<Recv<T>> recv;
  std::vector<Grid<T>> grids;
  std::vector<Helio<T>> helios;
  std::vector<T> factor;  // per heliostat
};

template <class T>
V<T> v3(const float* p) {
  return mk<T>(T(p[0]), T(p[1]), T(p[2]));
}

// Receiver set-up: RectangleReceiver::CInit (RectangleReceiver.cu:9-105),
// CylinderReceiver::CInit (CylinderReceiver.cu:4-15).
template <class T>
void recv_init(Recv<T>& r, int ppm) {
  r.pixel_length = T(1) / T(ppm);
  if (r.type == 1) {
    r.res_x = int(std::ceil(2 * M_PI * (double)r.size.x * (double)T(ppm)));
    r.res_y = int(r.size.y * T(ppm));
    return;
  }
  const V<T> s = r.size;
  const T h = T(2);
  switch (r.face) {
    case 0:
      r.local_normal = mk<T>(0, 0, 1);
      r.vert[0] = mk<T>(-s.x / h, -s.y / h, s.z / h);
      r.vert[1] = mk<T>(-s.x / h, s.y / h, s.z / h);
      r.vert[2] = mk<T>(s.x / h, s.y / h, s.z / h);
      r.vert[3] = mk<T>(s.x / h, -s.y / h, s.z / h);
      break;
    case 1:
      r.local_normal = mk<T>(1, 0, 0);
      r.vert[0] = mk<T>(s.x / h, -s.y / h, s.z / h);
      r.vert[1] = mk<T>(s.x / h, s.y / h, s.z / h);
      r.vert[2] = mk<T>(s.x / h, s.y / h, -s.z / h);
      r.vert[3] = mk<T>(s.x / h, -s.y / h, -s.z / h);
      break;
    case 2:
      r.local_normal = mk<T>(0, 0, -1);
      r.vert[0] = mk<T>(s.x / h, -s.y / h, -s.z / h);
      r.vert[1] = mk<T>(s.x / h, s.y / h, -s.z / h);
      r.vert[2] = mk<T>(-s.x / h, s.y / h, -s.z / h);
      r.vert[3] = mk<T>(-s.x / h, -s.y / h, -s.z / h);
      break;
    default:
      r.local_normal = mk<T>(-1, 0, 0);
      r.vert[0] = mk<T>(-s.x / h, -s.y / h, -s.z / h);
      r.vert[1] = mk<T>(-s.x / h, s.y / h, -s.z / h);
      r.vert[2] = mk<T>(-s.x / h, s.y / h, s.z / h);
      r.vert[3] = mk<T>(-s.x / h, -s.y / h, s.z / h);
      break;
  }
  r.normal = normalize(r.normal);
  for (auto& v : r.vert) v = rotate_yaw(v, r.local_normal, r.normal) + r.pos;
  r.focus = half_of(r.vert[0] + r.vert[2]);
  r.res_x = int(r.size.x * T(ppm));
  r.res_y = int(r.size.y * T(ppm));
}

// Receiver::getFocusCenter (RectangleReceiver.cu:103-105, CylinderReceiver.cu:18-31).
template <class T>
V<T> focus_of(const Recv<T>& r, V<T> hp) {
  if (r.type == 0) return r.focus;
  T lx = hp.x - r.pos.x, lz = hp.z - r.pos.z;
  if (lx * lx + lz * lz <= r.size.x * r.size.x) return r.pos;
  V<T> d = normalize(hp - r.pos);
  T radius = r.size.x / std::sqrt(d.x * d.x + d.z * d.z);
  return mk<T>(r.pos.x + d.x * radius, r.pos.y, r.pos.z + d.z * radius);
}

// Heliostat::CSetNormal + CSetWorldVertex (Heliostat.cu:15-40) with the
// focus-flat focal-length reset (FocusFlatRectangleHelio.cu:333-339).
template <class T>
void helio_orient(Helio<T>& h, V<T> focus, V<T> sun) {
  if (h.type == 1 && h.focus_length < T(0)) h.focus_length = length(focus - h.pos);
  V<T> refl = normalize(focus - h.pos);
  h.normal = normalize(refl - sun);
  const V<T> s = h.size;
  h.vertex[0] = mk<T>(-s.x / 2, s.y / 2, -s.z / 2);
  h.vertex[1] = mk<T>(0, 0, s.z) + h.vertex[0];
  h.vertex[2] = mk<T>(s.x, 0, s.z) + h.vertex[0];
  h.vertex[3] = mk<T>(s.x, 0, 0) + h.vertex[0];
  for (auto& v : h.vertex) v = rotate(v, h.normal, false) + h.pos;
}

// Sub-heliostat lengths and micro-facet lattice (RectangleHelio.cu:84-104,
// FocusFlatRectangleHelio.cu:68-82).  The lattice counts are evaluated in
// float in both precisions: they decide which micro-facets exist (4 m /
// 0.05 m is 80 facets in float, 79 in double), and the FP64 oracle traces
// the same facets as the float one, only in double.
template <class T>
void helio_lattice(Helio<T>& h) {
  h.len_x = (h.size.z - h.gap_y * T(h.rows - 1)) / T(h.rows);
  h.len_y = (h.size.x - h.gap_x * T(h.cols - 1)) / T(h.cols);
  const float lx = ((float)h.size.z - (float)h.gap_y * float(h.rows - 1)) / float(h.rows);
  const float ly = ((float)h.size.x - (float)h.gap_x * float(h.cols - 1)) / float(h.cols);
  h.sub_rows = int(lx / (float)h.pixel_length);
  h.sub_cols = int(ly / (float)h.pixel_length);
  h.n_facets = h.rows * h.cols * h.sub_rows * h.sub_cols;
}

// CGetSubHeliostatVertexes (RectangleHelio.cu:14-18; FocusFlatRectangleHelio.cu:123-227).
template <class T>
void helio_subverts(Helio<T>& h, std::vector<V<T>>& out) {
  if (h.type == 0) {
    out.push_back(h.vertex[0]);
    out.push_back(h.vertex[1]);
    out.push_back(h.vertex[2]);
    return;
  }
  const T lx = h.len_x, ly = h.len_y;
  const V<T> corners[3] = {mk<T>(-ly / 2, 0, lx / 2), mk<T>(-ly / 2, 0, -lx / 2), mk<T>(ly / 2, 0, -lx / 2)};
  const int n = h.rows * h.cols;
  h.lc.assign(n, mk<T>(0, 0, 0));
  h.ln.assign(n, mk<T>(0, 0, 0));
  for (int r = 0; r < h.rows; ++r)
    for (int c = 0; c < h.cols; ++c) {
      const int id = r * h.cols + c;
      if (h.read_method == -1) {
        V<T> cen = mk<T>(T(c) * (h.gap_x + ly) - h.size.x / 2 + ly / 2, h.size.y / 2,
                         T(r) * (h.gap_y + lx) - h.size.z / 2 + lx / 2);
        cen.y += (cen.x * cen.x + cen.z * cen.z) / (T(4) * h.focus_length);
        h.lc[id] = cen;
        h.ln[id] = normalize(mk<T>(T(-1) / (T(2) * h.focus_length) * cen.x, T(1),
                                   T(-1) / (T(2) * h.focus_length) * cen.z));
      } else {
        h.lc[id] = h.file_c[id];
        h.ln[id] = normalize(h.file_n[id]);
      }
      for (const auto& k : corners) {
        V<T> p = rotate(k, h.ln[id], true) + h.lc[id];
        out.push_back(rotate(p, h.normal, true) + h.pos);
      }
    }
}

// RectangleGrid::Cinit + CGridHelioMatch + boxIntersect (RectangleGrid.cu:8-117).
template <class T>
void grid_match(Grid<T>& g, const std::vector<Helio<T>>& hs) {
  g.nx = int(std::ceil(g.size.x / g.inter.x));
  g.ny = int(std::ceil(g.size.y / g.inter.y));
  g.nz = int(std::ceil(g.size.z / g.inter.z));
  const long long ncell = (long long)g.nx * g.ny * g.nz;
  std::vector<std::vector<int>> lists(ncell);
  int start_sub = 0;
  for (int i = g.start; i < g.start + g.count; ++i) {
    const auto& h = hs[i];
    T radius = length(h.size) / T(2);
    V<T> lo = cwise_div(minus_s(h.pos, radius) - g.pos, g.inter);
    V<T> hi = cwise_div(plus_s(h.pos, radius) - g.pos, g.inter);
    int lx = int(lo.x), ly = int(lo.y), lz = int(lo.z), hx = int(hi.x), hy = int(hi.y), hz = int(hi.z);
    for (int x = std::max(0, lx); x <= std::min(g.nx - 1, hx); ++x)
      for (int y = std::max(0, ly); y <= std::min(g.ny - 1, hy); ++y)
        for (int z = std::max(0, lz); z <= std::min(g.nz - 1, hz); ++z)
          for (int k = 0; k < h.n_sub; ++k) lists[((long long)x * g.ny + y) * g.nz + z].push_back(start_sub + k);
    start_sub += h.n_sub;
  }
  g.index.assign(ncell + 1, 0);
  g.match.clear();
  for (long long c = 0; c < ncell; ++c) {
    g.index[c + 1] = g.index[c] + (int)lists[c].size();
    g.match.insert(g.match.end(), lists[c].begin(), lists[c].end());
  }
}

// SceneProcessor::set_grid_receiver_heliostat_content (SceneProcessor.cpp:13-39)
// and the per-trace vertex tables (QuasiMonteCarloRayTracer.cpp:182-209).
template <class T>
std::unique_ptr<Scene<T>> build(const Desc& d) {
  auto s = std::make_unique<Scene<T>>();
  s->sun = mk<T>(T(d.sun_dir[0]), T(d.sun_dir[1]), T(d.sun_dir[2]));
  s->dni = T(d.dni);
  s->rho = T(d.rho);
  s->per_group = d.per_group;
  for (int i = 0; i < d.n_recv; ++i) {
    Recv<T> r{};
    r.type = d.recv_type[i];
    r.face = d.recv_face[i];
    r.pos = v3<T>(d.recv_pos + 3 * i);
    r.size = v3<T>(d.recv_size + 3 * i);
    r.normal = v3<T>(d.recv_norm + 3 * i);
    s->recv.push_back(r);
  }
  for (int i = 0; i < d.n_helio; ++i) {
    Helio<T> h{};
    h.type = d.h_type[i];
    h.grid = d.h_grid[i];
    h.pos = v3<T>(d.h_pos + 3 * i);
    h.size = v3<T>(d.h_size + 3 * i);
    h.gap_x = T(d.h_gap[2 * i]);
    h.gap_y = T(d.h_gap[2 * i + 1]);
    h.rows = d.h_matrix[2 * i];
    h.cols = d.h_matrix[2 * i + 1];
    h.n_sub = h.type == 1 ? h.rows * h.cols : 1;
    h.focus_length = h.type == 1 ? T(d.h_surface[6 * i]) : T(-1);
    h.read_method = h.type == 1 ? int(d.h_surface[6 * i + 1]) : -1;
    if (d.h_local_off && d.h_local_off[i] >= 0)
      for (int k = 0; k < h.rows * h.cols; ++k) {
        h.file_c.push_back(v3<T>(d.local_centers + 3 * (d.h_local_off[i] + k)));
        h.file_n.push_back(v3<T>(d.local_normals + 3 * (d.h_local_off[i] + k)));
      }
    s->helios.push_back(h);
  }
  const float ppm_f = 1.0f / d.recv_px;  // int(1.0f / receiver_pixel_length), SceneProcessor.cpp:21
  const int ppm = int(ppm_f);
  for (int gi = 0; gi < d.n_grid; ++gi) {
    Grid<T> g{};
    g.pos = v3<T>(d.grid_pos + 3 * gi);
    g.size = v3<T>(d.grid_size + 3 * gi);
    g.inter = v3<T>(d.grid_inter + 3 * gi);
    g.start = d.grid_start[gi];
    g.count = d.grid_n[gi];
    g.recv = d.grid_recv[gi];
    grid_match(g, s->helios);
    Recv<T>& r = s->recv[g.recv];
    recv_init(r, ppm);
    for (int i = g.start; i < g.start + g.count; ++i) {
      auto& h = s->helios[i];
      h.pixel_length = T(d.helio_px);
      helio_orient(h, focus_of(r, h.pos), s->sun);
    }
    s->grids.push_back(std::move(g));
  }
  for (auto& g : s->grids) {
    int sub = 0;
    for (int i = g.start; i < g.start + g.count; ++i) {
      auto& h = s->helios[i];
      h.sub_begin = sub;
      sub += h.n_sub;
      helio_lattice(h);
      helio_subverts(h, g.verts);
    }
  }
  s->factor.resize(s->helios.size());
  for (size_t i = 0; i < s->helios.size(); ++i) {
    const auto& h = s->helios[i];
    const auto& r = s->recv[s->grids[h.grid].recv];
    // QuasiMonteCarloRayTracer.cpp:58-60
    T ratio = h.pixel_length / r.pixel_length;
    s->factor[i] = s->dni * ratio * ratio * s->rho / T(s->per_group);
  }
  return s;
}

// Micro-facet centre and normal (RectangleHelio.cu:54-80; FocusFlatRectangleHelio.cu:12-64).
template <class T>
void facet(const Helio<T>& h, int f, V<T>& o, V<T>& n) {
  const int per_row = h.cols * h.sub_cols;
  int row = f / per_row, col = f % per_row;
  if (h.type == 0) {
    const int br = row / h.sub_rows, bc = col / h.sub_cols;
    V<T> c;
    c.x = T(col) * h.pixel_length + T(bc) * h.gap_x + h.pixel_length / 2 - h.size.x / 2;
    c.y = h.size.y / 2;
    c.z = T(row) * h.pixel_length + T(br) * h.gap_y + h.pixel_length / 2 - h.size.z / 2;
    o = rotate(c, h.normal, false) + h.pos;
    n = h.normal;
    return;
  }
  const int block = (row / h.sub_rows) * h.cols + col / h.sub_cols;
  row %= h.sub_rows;
  col %= h.sub_cols;
  V<T> lp = mk<T>((T(col) + T(0.5)) * h.pixel_length - h.len_y / 2, T(0),
                  (T(row) + T(0.5)) * h.pixel_length - h.len_x / 2);
  lp = rotate(lp, h.ln[block], true) + h.lc[block];
  n = rotate(h.ln[block], h.normal, true);
  o = rotate(lp, h.normal, true) + h.pos;
}

// rectGridDDA::collision / intersect (rectGridDDA.cu:7-119, helpers rectGridDDA.cuh:15-32).
template <class T> T abs_div(T den, T num) {
  if ((double)num <= EPS && (double)num >= -EPS) return T(INT_MAX);
  return std::fabs(den / num);
}
template <class T> bool less_e(T a, T b) { return (double)a < (double)b - EPS; }
template <class T> bool equal_e(T a, T b) { return (double)a < (double)b + EPS && (double)a > (double)b - EPS; }

struct WalkFlags {
  long long capped = 0;
};

template <class T>
bool walk(const Grid<T>& g, int own_begin, int own_n, V<T> o, V<T> d, Census* cz, WalkFlags& wf) {
  V<T> rel = o - g.pos;
  V<T> cf = cwise_div(rel, g.inter);
  int cx = int(cf.x), cy = int(cf.y), cz_ = int(cf.z);
  const int sx = d.x >= 0 ? 1 : -1, sy = d.y >= 0 ? 1 : -1, sz = d.z >= 0 ? 1 : -1;
  auto tmax0 = [](T dir, T inter, int idx, T pos) { return std::fabs(T(idx + (dir >= 0)) * inter - pos); };
  T tx = abs_div(tmax0(d.x, g.inter.x, cx, rel.x), d.x);
  T ty = abs_div(tmax0(d.y, g.inter.y, cy, rel.y), d.y);
  T tz = abs_div(tmax0(d.z, g.inter.z, cz_, rel.z), d.z);
  const T dx = abs_div(g.inter.x, d.x), dy = abs_div(g.inter.y, d.y), dz = abs_div(g.inter.z, d.z);
  const int cap = g.nx + g.ny + g.nz + 2;
  for (int it = 0; it < cap; ++it) {
    if (cx < 0 || cx >= g.nx || cy < 0 || cy >= g.ny || cz_ < 0 || cz_ >= g.nz) return false;
    if (cz) ++cz->cells;
    const int cell = cx * g.ny * g.nz + cy * g.nz + cz_;
    for (int k = g.index[cell]; k < g.index[cell + 1]; ++k) {
      const int s = g.match[k];
      if (s >= own_begin && s < own_begin + own_n) continue;
      T t, u, v;
      if (parallelogram(o, d, g.verts[3 * s + 1], g.verts[3 * s], g.verts[3 * s + 2], t, u, v, cz)) return true;
    }
    bool fx = false, fy = false, fz = false;
    if (less_e(tx, ty)) {
      if (less_e(tx, tz) || equal_e(tx, tz)) cx += sx, fx = true;
      if (less_e(tz, tx) || equal_e(tx, tz)) cz_ += sz, fz = true;
    } else if (less_e(ty, tx)) {
      if (less_e(ty, tz) || equal_e(ty, tz)) cy += sy, fy = true;
      if (less_e(tz, ty) || equal_e(ty, tz)) cz_ += sz, fz = true;
    } else {
      if (less_e(tx, tz) || equal_e(tx, tz)) cx += sx, cy += sy, fx = fy = true;
      if (less_e(tz, tx) || equal_e(tx, tz)) cz_ += sz, fz = true;
    }
    if (!(fx || fy || fz)) {
      ++wf.capped;
      return false;
    }
    tx += fx ? dx : T(0);
    ty += fy ? dy : T(0);
    tz += fz ? dz : T(0);
  }
  ++wf.capped;
  return false;
}

// CylinderReceiver::GIntersect (CylinderReceiver.cuh:39-89); the acos
// argument is clamped to [-1, 1] (the reference prints an error and lets
// NaN through when rounding pushes it outside).
template <class T>
bool cylinder_hit(const Recv<T>& r, V<T> o, V<T> d, T& t, T& u, T& v) {
  T lx = o.x - r.pos.x, lz = o.z - r.pos.z;
  if (lx * lx + lz * lz <= r.size.x * r.size.x) return false;
  T rox = r.pos.x - o.x, roz = r.pos.z - o.z;
  T il = inv_sqrt(d.x * d.x + d.z * d.z);
  T tp = rox * (d.x * il) + roz * (d.z * il);
  T delta = (rox * rox + roz * roz) - tp * tp;
  T r2 = r.size.x * r.size.x;
  if ((double)tp < -EPS || delta > r2) return false;
  T tplus = delta <= T(0) ? r.size.x : std::sqrt(r2 - delta);
  t = (tp - tplus) / std::sqrt(d.x * d.x + d.z * d.z);
  V<T> ip = d * t + o;
  u = (ip.y - r.pos.y) / r.size.y + T(0.5);
  if (u < T(0) || u > T(1)) return false;
  T ex = ip.x - r.pos.x, ez = ip.z - r.pos.z;
  T ie = inv_sqrt(ex * ex + ez * ez);
  T cx = ex * ie, sy = ez * ie;
  cx = std::min(std::max(cx, T(-1)), T(1));
  v = T((double)std::acos(cx) / (2 * M_PI));
  if (sy < 0) v = T(1) - v;
  return true;
}

// eta_aAlpha / calEnergy (receiverIntersectionUtil.cuh:17-34).
template <class T>
T energy(T dist, V<T> d, V<T> n, T factor) {
  T eta = dist <= T(1000) ? T(0.99331f) - T(0.0001176f) * dist + T(1.97f) * T(1e-8f) * dist * dist
                          : std::exp(T(-0.0001106f) * dist);
  return std::fabs(dot(d, n)) * eta * factor;
}

// ---------------------------------------------------------------------------
struct TraceArgs {
  const int* ids;
  int n_ids;
  const float* pool_dirs;     // P float3
  const float* pool_pert;     // P float3
  int pool_size;
  const int* offsets;         // concatenated num_facets+1 per heliostat
  const long long* offset_base;  // per heliostat, index into offsets
  int light_begin, light_end;
  int facet_stride;           // trace facets f with f % stride == phase
  int facet_phase;
  // outputs (may be null)
  double* images;             // concatenated receiver images
  const long long* image_base;
  double* power;              // per heliostat
  long long* counters;        // 12: rays, shadowed, blocked, missed, hit, clamped, capped, cells, det, u, v, t
  // per-ray records for one heliostat
  int rec_id, rec_facet_begin, rec_facet_end;
  int* records;
  int threads;
  int record_only;            // with records: trace only heliostat rec_id's facets [rec_facet_begin, rec_facet_end)
};

template <class T>
void trace(const Scene<T>& s, const TraceArgs& a) {
  const int P = a.pool_size;
  V<T> nsun = -s.sun;
  long long totals[12] = {0};
  const long long total_pix = a.images ? a.image_base[s.recv.size()] : 0;
#ifdef _OPENMP
  if (a.threads > 0) omp_set_num_threads(a.threads);
#endif
#pragma omp parallel
  {
    std::vector<double> img(a.images ? total_pix : 0, 0.0);
    std::vector<double> pw(s.helios.size(), 0.0);
    long long cnt[12] = {0};
    Census cz;
    WalkFlags wf;
    for (int ti = 0; ti < a.n_ids; ++ti) {
      const int hid = a.ids[ti];
      const Helio<T>& h = s.helios[hid];
      const Grid<T>& g = s.grids[h.grid];
      const Recv<T>& r = s.recv[g.recv];
      const int* off = a.offsets + a.offset_base[hid];
      const T factor = s.factor[hid];
      const bool only = a.records && a.record_only && hid == a.rec_id;
      const int f_begin = only ? std::max(0, a.rec_facet_begin) : 0;
      const int f_end = only ? std::min(h.n_facets, a.rec_facet_end) : h.n_facets;
#pragma omp for schedule(dynamic, 64) nowait
      for (int f = f_begin; f < f_end; ++f) {
        if (a.facet_stride > 1 && f % a.facet_stride != a.facet_phase) continue;
        V<T> o, n0;
        facet(h, f, o, n0);
        const int g0 = off[f];
        const int g1 = off[(f + 1) % P];
        for (int l = a.light_begin; l < a.light_end; ++l) {
          ++cnt[0];
          const int ai = (g0 + l) % P;
          V<T> dir = rotate(v3<T>(a.pool_dirs + 3 * ai), nsun, false);
          int code;
          if (walk(g, h.sub_begin, h.n_sub, o, dir, &cz, wf)) {
            code = -1;
            ++cnt[1];
          } else {
            const int bi = (g1 + l) % P;
            V<T> n = normalize(rotate(v3<T>(a.pool_pert + 3 * bi), n0, false));
            V<T> rd = normalize(reflect(-dir, n));
            if (walk(g, h.sub_begin, h.n_sub, o, rd, &cz, wf)) {
              code = -2;
              ++cnt[2];
            } else {
              T t, u, v;
              bool hit = r.type == 0 ? parallelogram(o, rd, r.vert[0], r.vert[1], r.vert[3], t, u, v, nullptr)
                                     : cylinder_hit(r, o, rd, t, u, v);
              if (!hit) {
                code = -3;
                ++cnt[3];
              } else {
                T e = energy(t, rd, n, factor);
                int row = int(u * T(r.res_y)), col = int(v * T(r.res_x));
                if (row >= r.res_y || col >= r.res_x || row < 0 || col < 0) {
                  row = std::min(std::max(row, 0), r.res_y - 1);
                  col = std::min(std::max(col, 0), r.res_x - 1);
                  ++cnt[5];
                }
                code = row * r.res_x + col;
                ++cnt[4];
                if (a.images) img[a.image_base[g.recv] + code] += (double)e;
                pw[hid] += (double)e;
              }
            }
          }
          if (a.records && hid == a.rec_id && f >= a.rec_facet_begin && f < a.rec_facet_end)
            a.records[(long long)(f - a.rec_facet_begin) * (a.light_end - a.light_begin) + (l - a.light_begin)] = code;
        }
      }
    }
    cnt[6] = wf.capped;
    cnt[7] = cz.cells;
    cnt[8] = cz.tests_det;
    cnt[9] = cz.tests_u;
    cnt[10] = cz.tests_v;
    cnt[11] = cz.tests_t;
#pragma omp critical
    {
      if (a.images)
        for (long long i = 0; i < total_pix; ++i) a.images[i] += img[i];
      if (a.power)
        for (size_t i = 0; i < pw.size(); ++i) a.power[i] += pw[i];
      for (int k = 0; k < 12; ++k) totals[k] += cnt[k];
    }
  }
  if (a.counters)
    for (int k = 0; k < 12; ++k) a.counters[k] += totals[k];
}

// ---------------------------------------------------------------------------
// Trimmed-mean smoother (Tool/Smoother/ImageSmoother.cu:13-64, heap.cuh:16-225).
struct HeapF {
  float* e;
  int num, cap;
  bool is_max;
  bool cmp(float a, float b) const { return is_max ? a > b : a < b; }
  bool full() const { return num == cap; }
  bool empty() const { return num == 1; }
  float top() const { return empty() ? 0.0f : e[1]; }
  void insert(float x) {
    if (full()) return;
    int i = num++;
    for (; i != 1 && cmp(x, e[i / 2]); i /= 2) e[i] = e[i / 2];
    e[i] = x;
  }
  void replace_top(float x) {
    if (empty()) return;
    int i = 1;
    while (2 * i < num) {
      int c = (2 * i + 1 >= num || cmp(e[2 * i], e[2 * i + 1])) ? 2 * i : 2 * i + 1;
      if (cmp(e[c], x)) {
        e[i] = e[c];
        i = c;
      } else {
        break;
      }
    }
    e[i] = x;
  }
  float sum() const {
    float s = 0.0f;
    for (int i = 1; i < num; ++i) s += e[i];
    return s;
  }
};

void smooth(const float* in, float* out, int w, int h, int radius, float ratio) {
#pragma omp parallel for schedule(static)
  for (int y = 0; y < h; ++y) {
    std::vector<float> a, b;
    for (int x = 0; x < w; ++x) {
      int x0 = std::max(x - radius, 0), y0 = std::max(y - radius, 0);
      int x1 = std::min(x + radius, w - 1), y1 = std::min(y + radius, h - 1);
      int cnt = (x1 - x0 + 1) * (y1 - y0 + 1);
      int k = cnt * ratio;
      a.assign(k + 2, 0.0f);
      b.assign(k + 2, 0.0f);
      HeapF lo{a.data(), 1, k + 1, true}, hi{b.data(), 1, k + 1, false};
      float value = 0.0f;
      for (int r = y0; r <= y1; ++r)
        for (int c = x0; c <= x1; ++c) {
          float cur = in[(long long)r * w + c];
          value += cur;
          if (!lo.full()) {
            lo.insert(cur);
            hi.insert(cur);
          } else if (cur < lo.top()) {
            lo.replace_top(cur);
          } else if (cur > hi.top()) {
            hi.replace_top(cur);
          }
        }
      out[(long long)y * w + x] = (value - lo.sum() - hi.sum()) / float(cnt - 2 * k);
    }
  }
}

// ---------------------------------------------------------------------------
// Reference Buie sampler restated (Scene/SceneProcessor.cu:7-81, :204-239).
struct Buie {
  std::vector<float> cdf_x, cdf_y, k;
  float less_465, gamma, A, B, C;
};

Buie buie_table(float csr, int n) {
  Buie t;
  const float up = 4.65f;
  const float kappa = 0.9f * logf(13.5f * csr) * powf(csr, -0.3f);
  const float gamma = 2.2f * logf(0.52f * csr) * powf(csr, 0.43f) - 0.1f;
  auto tail = [&](float th) { return expf(kappa) / (gamma + 1) * powf(th, gamma + 1); };
  auto core = [](float th) { return cosf(0.326f * th) / cosf(0.308f * th); };
  const float i_465_930 = tail(9.3f) - tail(up);
  t.cdf_x.assign(n + 1, 0.0f);
  t.cdf_y.assign(n + 1, 0.0f);
  t.k.assign(n, 0.0f);
  const float li = up / float(n);
  float x = 0.0f, pre = core(x);
  for (int i = 1; i <= n; ++i) {
    x += li;
    float cur = core(x);
    float area = (cur + pre) / 2.0f * li;
    t.cdf_x[i] = x;
    t.cdf_y[i] = area + t.cdf_y[i - 1];
    t.k[i - 1] = li / area;
    pre = cur;
  }
  t.less_465 = t.cdf_y[n];
  t.gamma = gamma;
  t.A = t.less_465 + i_465_930;
  t.B = (gamma + 1) / expf(kappa);
  t.C = powf(up, gamma + 1);
  return t;
}

float buie_theta(const Buie& b, float uniform) {
  float u = uniform * b.A;
  const int n = (int)b.k.size();
  if (u < b.less_465) {
    int left = 0, right = n, id;
    for (;;) {
      if (left > right) {
        id = right;
        break;
      }
      int mid = (left + right) >> 1;
      if (u > b.cdf_y[mid]) left = mid + 1;
      else if (u < b.cdf_y[mid]) right = mid - 1;
      else {
        id = mid;
        break;
      }
    }
    u = (u - b.cdf_y[id]) * b.k[id] + b.cdf_x[id];
    u = atanf(sqrtf(u / 4.65f) * 0.5016916f);
  } else {
    u = powf((u - b.less_465) * b.B + b.C, 1 / (b.gamma + 1));
    float ri2 = 0.5016916f * 0.5016916f, ro2 = 1.340874f * 1.340874f;
    u = atanf(sqrtf(ro2 + (u - 4.65f) / 4.65f * (ro2 - ri2)));
  }
  return u / 100.0f;
}

// Scrambled Sobol points: a restatement of B. Burley, "Practical Hash-based
// Owen Scrambling", JCGT 9(4) 2020 (the build's own generator, checked here
// bit for bit).
uint32_t rev(uint32_t x) {
  uint32_t r = 0;
  for (int i = 0; i < 32; ++i) r |= ((x >> i) & 1u) << (31 - i);
  return r;
}
uint32_t mix(uint32_t x) {
  x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
  return x;
}
uint32_t hcomb(uint32_t s, uint32_t v) { return s ^ (v + (s << 6) + (s >> 2)); }
uint32_t owen(uint32_t x, uint32_t seed) {
  x = rev(x);
  x += seed;
  x ^= x * 0x6c50b47cu;
  x ^= x * 0xb82f1e52u;
  x ^= x * 0xc7afe638u;
  x ^= x * 0x8d22f6e6u;
  return rev(x);
}
uint32_t sobol1(uint32_t i) {
  uint32_t r = 0, v = 0x80000000u;
  while (i) {
    if (i & 1u) r ^= v;
    i >>= 1;
    v ^= v >> 1;
  }
  return r;
}
void sobol2(uint32_t index, uint32_t seed, uint32_t& x, uint32_t& y) {
  uint32_t sh = owen(index, mix(seed));
  x = owen(rev(sh), mix(hcomb(seed, 0u)));
  y = owen(sobol1(sh), mix(hcomb(seed, 1u)));
}

}  // namespace oracle

// ---------------------------------------------------------------------------
extern "C" {

struct oracle_handle {
  std::unique_ptr<oracle::Scene<float>> f;
  std::unique_ptr<oracle::Scene<double>> d;
};

oracle_handle* oracle_create(const oracle::Desc* desc, int precision) {
  auto* h = new oracle_handle();
  if (precision == 64) h->d = oracle::build<double>(*desc);
  else h->f = oracle::build<float>(*desc);
  return h;
}

void oracle_free(oracle_handle* h) { delete h; }

void oracle_counts(oracle_handle* h, int* out3) {
  auto put = [&](auto& s) {
    out3[0] = (int)s.recv.size();
    out3[1] = (int)s.grids.size();
    out3[2] = (int)s.helios.size();
  };
  if (h->f) put(*h->f);
  else put(*h->d);
}

// Receiver: type, res_x, res_y; floats: pixel_length, 12 vertices, normal3, focus3.
void oracle_receiver(oracle_handle* h, int i, int* ints3, double* vals19) {
  auto put = [&](auto& s) {
    const auto& r = s.recv[i];
    ints3[0] = r.type;
    ints3[1] = r.res_x;
    ints3[2] = r.res_y;
    vals19[0] = r.pixel_length;
    for (int k = 0; k < 4; ++k) vals19[1 + 3 * k] = r.vert[k].x, vals19[2 + 3 * k] = r.vert[k].y, vals19[3 + 3 * k] = r.vert[k].z;
    vals19[13] = r.normal.x, vals19[14] = r.normal.y, vals19[15] = r.normal.z;
    vals19[16] = r.focus.x, vals19[17] = r.focus.y, vals19[18] = r.focus.z;
  };
  if (h->f) put(*h->f);
  else put(*h->d);
}

// Heliostat: type, grid, n_facets, n_sub, sub_begin; doubles: normal3, focus_length, factor.
void oracle_heliostat(oracle_handle* h, int i, int* ints5, double* vals5) {
  auto put = [&](auto& s) {
    const auto& x = s.helios[i];
    ints5[0] = x.type;
    ints5[1] = x.grid;
    ints5[2] = x.n_facets;
    ints5[3] = x.n_sub;
    ints5[4] = x.sub_begin;
    vals5[0] = x.normal.x, vals5[1] = x.normal.y, vals5[2] = x.normal.z;
    vals5[3] = x.focus_length;
    vals5[4] = s.factor[i];
  };
  if (h->f) put(*h->f);
  else put(*h->d);
}

// Grid: cells3, nnz, n_sub_vertices.
void oracle_grid(oracle_handle* h, int i, int* ints5) {
  auto put = [&](auto& s) {
    const auto& g = s.grids[i];
    ints5[0] = g.nx, ints5[1] = g.ny, ints5[2] = g.nz;
    ints5[3] = (int)g.match.size();
    ints5[4] = (int)g.verts.size() / 3;
  };
  if (h->f) put(*h->f);
  else put(*h->d);
}

void oracle_grid_csr(oracle_handle* h, int i, int* index, int* match) {
  auto put = [&](auto& s) {
    const auto& g = s.grids[i];
    std::copy(g.index.begin(), g.index.end(), index);
    std::copy(g.match.begin(), g.match.end(), match);
  };
  if (h->f) put(*h->f);
  else put(*h->d);
}

void oracle_grid_vertices(oracle_handle* h, int i, double* xyz) {
  auto put = [&](auto& s) {
    const auto& g = s.grids[i];
    for (size_t k = 0; k < g.verts.size(); ++k) xyz[3 * k] = g.verts[k].x, xyz[3 * k + 1] = g.verts[k].y, xyz[3 * k + 2] = g.verts[k].z;
  };
  if (h->f) put(*h->f);
  else put(*h->d);
}

void oracle_facets(oracle_handle* h, int i, double* origins, double* normals) {
  auto put = [&](auto& s) {
    const auto& x = s.helios[i];
    for (int f = 0; f < x.n_facets; ++f) {
      using T = decltype(x.pos.x);
      oracle::V<T> o, n;
      oracle::facet(x, f, o, n);
      origins[3 * f] = o.x, origins[3 * f + 1] = o.y, origins[3 * f + 2] = o.z;
      normals[3 * f] = n.x, normals[3 * f + 1] = n.y, normals[3 * f + 2] = n.z;
    }
  };
  if (h->f) put(*h->f);
  else put(*h->d);
}

void oracle_trace(oracle_handle* h, const oracle::TraceArgs* a) {
  if (h->f) oracle::trace(*h->f, *a);
  else oracle::trace(*h->d, *a);
}

// Single-ray grid walk, for unit checks: returns 1 on a hit.
int oracle_walk(oracle_handle* h, int grid, int own_begin, int own_n, const double* o, const double* d) {
  oracle::WalkFlags wf;
  if (h->f) {
    oracle::V<float> oo{(float)o[0], (float)o[1], (float)o[2]}, dd{(float)d[0], (float)d[1], (float)d[2]};
    return oracle::walk(h->f->grids[grid], own_begin, own_n, oo, dd, nullptr, wf) ? 1 : 0;
  }
  oracle::V<double> oo{o[0], o[1], o[2]}, dd{d[0], d[1], d[2]};
  return oracle::walk(h->d->grids[grid], own_begin, own_n, oo, dd, nullptr, wf) ? 1 : 0;
}

// Receiver intersection of one ray (float arithmetic): returns 1 on a hit, tuv = (t, u, v).
int oracle_receiver_hit(oracle_handle* h, int recv, const float* o, const float* d, float* tuv) {
  const auto& r = h->f->recv[recv];
  oracle::V<float> oo{o[0], o[1], o[2]}, dd{d[0], d[1], d[2]};
  float t = 0, u = 0, v = 0;
  bool hit = r.type == 0 ? oracle::parallelogram(oo, dd, r.vert[0], r.vert[1], r.vert[3], t, u, v, nullptr)
                         : oracle::cylinder_hit(r, oo, dd, t, u, v);
  tuv[0] = t, tuv[1] = u, tuv[2] = v;
  return hit ? 1 : 0;
}

void oracle_smooth(const float* in, float* out, int w, int h, int radius, float ratio) {
  oracle::smooth(in, out, w, h, radius, ratio);
}

// Buie inverse CDF of `n` uniforms with the reference's tables.
void oracle_buie(float csr, int groups, const float* uniforms, float* theta, int n) {
  oracle::Buie b = oracle::buie_table(csr, groups);
  for (int i = 0; i < n; ++i) theta[i] = oracle::buie_theta(b, uniforms[i]);
}

void oracle_buie_table(float csr, int groups, float* cdf_x, float* cdf_y, float* k, float* scalars5) {
  oracle::Buie b = oracle::buie_table(csr, groups);
  std::copy(b.cdf_x.begin(), b.cdf_x.end(), cdf_x);
  std::copy(b.cdf_y.begin(), b.cdf_y.end(), cdf_y);
  std::copy(b.k.begin(), b.k.end(), k);
  scalars5[0] = b.less_465, scalars5[1] = b.gamma, scalars5[2] = b.A, scalars5[3] = b.B, scalars5[4] = b.C;
}

void oracle_sobol2(uint32_t seed, uint32_t first, int n, uint32_t* xy) {
  for (int i = 0; i < n; ++i) oracle::sobol2(first + (uint32_t)i, seed, xy[2 * i], xy[2 * i + 1]);
}

void oracle_facet_offsets(uint32_t seed, uint32_t heliostat, int n, uint32_t pool, int* out) {
  uint32_t base = oracle::mix(seed ^ 0x9e3779b9u);
  for (int i = 0; i < n; ++i) {
    uint32_t h = oracle::mix(oracle::hcomb(oracle::hcomb(base, heliostat), (uint32_t)i));
    out[i] = (int)(((uint64_t)h * pool) >> 32);
  }
}

uint32_t oracle_mix32(uint32_t x) { return oracle::mix(x); }

}  // extern "C"

// ---------------------------------------------------------------------------
// Stand-alone probes of single reference routines, for the known-answer
// checks of the reference's gtest suites (float arithmetic).
extern "C" {

// One heliostat with an explicit normal (no focus/sun step): lattice,
// sub-heliostat table and micro-facets.  counts2 = (n_facets, n_sub).
int oracle_probe_heliostat(int type, const float* size3, const float* gap2, const int* matrix2, float px,
                           const float* normal3, const float* pos3, float focus_length, int cap, float* origins,
                           float* normals, float* subverts, float* local_centers, float* local_normals,
                           int* counts2) {
  using namespace oracle;
  Helio<float> h{};
  h.type = type;
  h.size = v3<float>(size3);
  h.gap_x = gap2[0];
  h.gap_y = gap2[1];
  h.rows = matrix2[0];
  h.cols = matrix2[1];
  h.n_sub = type == 1 ? h.rows * h.cols : 1;
  h.pixel_length = px;
  h.normal = v3<float>(normal3);
  h.pos = v3<float>(pos3);
  h.focus_length = focus_length;
  h.read_method = -1;
  // Heliostat::CSetWorldVertex with the given normal (Heliostat.cu:25-40).
  const V<float> s = h.size;
  h.vertex[0] = mk<float>(-s.x / 2, s.y / 2, -s.z / 2);
  h.vertex[1] = mk<float>(0, 0, s.z) + h.vertex[0];
  h.vertex[2] = mk<float>(s.x, 0, s.z) + h.vertex[0];
  h.vertex[3] = mk<float>(s.x, 0, 0) + h.vertex[0];
  for (auto& v : h.vertex) v = rotate(v, h.normal, false) + h.pos;
  helio_lattice(h);
  std::vector<V<float>> sv;
  helio_subverts(h, sv);
  counts2[0] = h.n_facets;
  counts2[1] = h.n_sub;
  if (h.n_facets > cap) return -1;
  for (int f = 0; f < h.n_facets; ++f) {
    V<float> o, n;
    facet(h, f, o, n);
    origins[3 * f] = o.x, origins[3 * f + 1] = o.y, origins[3 * f + 2] = o.z;
    normals[3 * f] = n.x, normals[3 * f + 1] = n.y, normals[3 * f + 2] = n.z;
  }
  for (size_t k = 0; k < sv.size(); ++k) subverts[3 * k] = sv[k].x, subverts[3 * k + 1] = sv[k].y, subverts[3 * k + 2] = sv[k].z;
  for (size_t k = 0; k < h.lc.size(); ++k) {
    local_centers[3 * k] = h.lc[k].x, local_centers[3 * k + 1] = h.lc[k].y, local_centers[3 * k + 2] = h.lc[k].z;
    local_normals[3 * k] = h.ln[k].x, local_normals[3 * k + 1] = h.ln[k].y, local_normals[3 * k + 2] = h.ln[k].z;
  }
  return 0;
}

static oracle::Recv<float> probe_cylinder(const float* pos3, const float* size3) {
  oracle::Recv<float> r{};
  r.type = 1;
  r.pos = oracle::v3<float>(pos3);
  r.size = oracle::v3<float>(size3);
  return r;
}

int oracle_probe_cylinder_hit(const float* pos3, const float* size3, const float* o, const float* d, float* tuv) {
  auto r = probe_cylinder(pos3, size3);
  float t = 0, u = 0, v = 0;
  bool hit = oracle::cylinder_hit(r, oracle::v3<float>(o), oracle::v3<float>(d), t, u, v);
  tuv[0] = t, tuv[1] = u, tuv[2] = v;
  return hit ? 1 : 0;
}

void oracle_probe_cylinder_focus(const float* pos3, const float* size3, const float* helio3, float* out3) {
  auto r = probe_cylinder(pos3, size3);
  auto f = oracle::focus_of(r, oracle::v3<float>(helio3));
  out3[0] = f.x, out3[1] = f.y, out3[2] = f.z;
}

void oracle_probe_cylinder_resolution(const float* size3, int ppm, int* out2) {
  float pos[3] = {0, 0, 0};
  auto r = probe_cylinder(pos, size3);
  oracle::recv_init(r, ppm);
  out2[0] = r.res_x, out2[1] = r.res_y;
}

// CGridHelioMatch for explicit heliostats (position, size, sub-heliostat count).
int oracle_probe_grid(const float* pos3, const float* size3, const float* inter3, int n, const float* hpos,
                      const float* hsize, const int* nsub, int cap, int* index, int* match, int* counts4) {
  using namespace oracle;
  Grid<float> g{};
  g.pos = v3<float>(pos3);
  g.size = v3<float>(size3);
  g.inter = v3<float>(inter3);
  g.start = 0;
  g.count = n;
  std::vector<Helio<float>> hs(n);
  for (int i = 0; i < n; ++i) {
    hs[i].pos = v3<float>(hpos + 3 * i);
    hs[i].size = v3<float>(hsize + 3 * i);
    hs[i].n_sub = nsub[i];
  }
  grid_match(g, hs);
  counts4[0] = g.nx, counts4[1] = g.ny, counts4[2] = g.nz, counts4[3] = (int)g.match.size();
  if ((int)g.index.size() > cap || (int)g.match.size() > cap) return -1;
  std::copy(g.index.begin(), g.index.end(), index);
  std::copy(g.match.begin(), g.match.end(), match);
  return 0;
}

}  // extern "C"
