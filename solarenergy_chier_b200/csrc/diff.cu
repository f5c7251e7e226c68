// Differentiable forward and hand-written adjoint of the tracer.
//
// Forward (diff.cpp drives it): the heliostats are prepared with their
// parameters -- aim point moved by (du, dv) along the receiver's aim axes,
// normal then turned by (a, b) radians about its frame's u and v axes --
// every ray is traced as in the plain path, each receiver hit deposits its
// energy bilinearly at its continuous pixel position (trace kernel output
// mode 2, which also records one hit bit per ray), the deposit D is smoothed
// by a separable Gaussian G (flux F = G * D) and L = sum (F - T)^2.
//
// Adjoint: with R = dL/dF = 2 (F - T) and P = G * R (G is symmetric, so
// dL/dD = P), a ray depositing energy e at pixel position (X, Y) contributes
//   dL/dtheta = e (dPb/dX dX/dtheta + dPb/dY dY/dtheta) + Pb de/dtheta,
// Pb the bilinear interpolation of P at (X, Y) -- the exact derivative of
// the discretised forward.  (X, Y) and e are differentiated forward-mode
// (value + 4 tangents) from the heliostat's parameters through its normal
// and frame, the facet position and normal, the slope-error normal, the
// reflection, the receiver intersection (implicitly: the hit point stays on
// the receiver surface) and the energy (cosine and atmospheric attenuation).
// Shadowing and blocking are treated as constants (indicators detached):
// only rays whose hit bit the forward set contribute, and no grid walk is
// repeated.  The receiver's own edges (a cylinder's silhouette, the image's
// first and last rows and a rectangle's columns) are handled by band
// estimates of their boundary terms.  The bias left is the change of loss
// from rays that cross a blocker's edge.
#include "diff.h"

#include "ray_geom.h"

namespace qm {
namespace {

constexpr int K = kDiffParams;
// Smallest |cos(incidence)| on the receiver of a ray whose interior
// derivative is used (about 84 degrees from the surface normal); grazing rays
// on a cylinder estimate its silhouette's boundary term instead.
constexpr float kGrazing = 0.1f;
// Width in pixels of the bands along the image edges whose rays estimate
// the edges' boundary terms.
constexpr float kEdgeBand = 1.0f;
constexpr float kTwoPi = 6.28318530717959f;

// ---- value + tangent arithmetic ----------------------------------------------
__device__ __forceinline__ Dual dc(float v) {
  Dual r;
  r.v = v;
#pragma unroll
  for (int k = 0; k < K; ++k) r.d[k] = 0.0f;
  return r;
}
__device__ __forceinline__ Dual dvar(float v, int k) {
  Dual r = dc(v);
  r.d[k] = 1.0f;
  return r;
}
__device__ __forceinline__ Dual operator+(Dual a, Dual b) {
  Dual r;
  r.v = a.v + b.v;
#pragma unroll
  for (int k = 0; k < K; ++k) r.d[k] = a.d[k] + b.d[k];
  return r;
}
__device__ __forceinline__ Dual operator-(Dual a, Dual b) {
  Dual r;
  r.v = a.v - b.v;
#pragma unroll
  for (int k = 0; k < K; ++k) r.d[k] = a.d[k] - b.d[k];
  return r;
}
__device__ __forceinline__ Dual operator-(Dual a) {
  Dual r;
  r.v = -a.v;
#pragma unroll
  for (int k = 0; k < K; ++k) r.d[k] = -a.d[k];
  return r;
}
__device__ __forceinline__ Dual operator*(Dual a, Dual b) {
  Dual r;
  r.v = a.v * b.v;
#pragma unroll
  for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
  return r;
}
__device__ __forceinline__ Dual operator*(Dual a, float s) {
  Dual r;
  r.v = a.v * s;
#pragma unroll
  for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * s;
  return r;
}
// 1 / sqrt(a)
__device__ __forceinline__ Dual drsqrt(Dual a) {
  const float r = rsqrtf(a.v);
  const float dr = -0.5f * r * r * r;
  Dual o;
  o.v = r;
#pragma unroll
  for (int k = 0; k < K; ++k) o.d[k] = dr * a.d[k];
  return o;
}

__device__ __forceinline__ Dual3 d3(float3 c) { return Dual3{dc(c.x), dc(c.y), dc(c.z)}; }
__device__ __forceinline__ float3 val(const Dual3& a) { return make_float3(a.x.v, a.y.v, a.z.v); }
__device__ __forceinline__ Dual3 operator+(const Dual3& a, const Dual3& b) { return Dual3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ Dual3 operator-(const Dual3& a, const Dual3& b) { return Dual3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ Dual3 operator-(const Dual3& a) { return Dual3{-a.x, -a.y, -a.z}; }
__device__ __forceinline__ Dual3 operator*(const Dual3& a, Dual s) { return Dual3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ Dual3 operator*(const Dual3& a, float s) { return Dual3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ Dual dot(const Dual3& a, const Dual3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ Dual3 cross(const Dual3& a, const Dual3& b) {
  return Dual3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ Dual3 normalize(const Dual3& a) { return a * drsqrt(dot(a, a)); }

// Frame (u, n, v) of a normal, as qm::make_frame (Util/global_function.cuh:19-36
// and the flipped focus-flat variant), with tangents.
struct DFrame {
  Dual3 u, n, v;
  bool identity;
};
__device__ __forceinline__ DFrame make_dframe(const Dual3& n, bool flip) {
  DFrame f;
  f.n = n;
  f.identity = qm_below_eps(fabsf(n.x.v)) && qm_below_eps(fabsf(n.z.v));
  if (f.identity) {
    f.u = d3(make_float3(1.f, 0.f, 0.f));
    f.v = d3(make_float3(0.f, 0.f, 1.f));
    return f;
  }
  f.u = normalize(cross(d3(make_float3(0.f, 1.f, 0.f)), n));
  f.v = normalize(cross(f.u, n));
  if (flip && n.z.v < 0) {
    f.u = -f.u;
    f.v = -f.v;
  }
  return f;
}
__device__ __forceinline__ Dual3 to_world(const DFrame& f, float3 d) {
  if (f.identity) return d3(d);
  return f.u * d.x + f.n * d.y + f.v * d.z;
}

// ---- preparation: normal and frame of every heliostat with tangents --------
__global__ void diff_prep_kernel(const PrepItem* items, int n, const DevTask* tasks, DiffTask* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const PrepItem it = items[i];
  const DevTask& T = tasks[it.task];
  // aim point a = focus + du aim_u + dv aim_v
  Dual3 a = d3(make_float3(it.focus.x + it.aim_u.x * it.aim_offset.x + it.aim_v.x * it.aim_offset.y,
                           it.focus.y + it.aim_u.y * it.aim_offset.x + it.aim_v.y * it.aim_offset.y,
                           it.focus.z + it.aim_u.z * it.aim_offset.x + it.aim_v.z * it.aim_offset.y));
  a.x.d[0] = it.aim_u.x;
  a.y.d[0] = it.aim_u.y;
  a.z.d[0] = it.aim_u.z;
  a.x.d[1] = it.aim_v.x;
  a.y.d[1] = it.aim_v.y;
  a.z.d[1] = it.aim_v.z;
  const Dual3 r = normalize(a - d3(T.pos));
  const Dual3 n0 = normalize(r - d3(it.sun_dir));
  const DFrame f0 = make_dframe(n0, false);
  const Dual3 nrm = normalize(n0 + f0.u * dvar(it.normal_offset.x, 2) + f0.v * dvar(it.normal_offset.y, 3));
  const DFrame hf = make_dframe(nrm, T.type == 1);
  DiffTask o;
  o.n = nrm;
  o.u = hf.u;
  o.fn = hf.n;
  o.v = hf.v;
  o.identity = hf.identity ? 1 : 0;
  out[it.task] = o;
}

// ---- adjoint ------------------------------------------------------------------
__device__ __forceinline__ float sample_p(const DevReceiver& R, int c, int r) {
  const int w = R.resolution.x, h = R.resolution.y;
  if (R.type == 1) c = c < 0 ? c + w : (c >= w ? c - w : c);
  if (c < 0 || c >= w || r < 0 || r >= h) return 0.0f;
  return __ldg(R.image + r * w + c);
}

// Bilinear interpolation of P at continuous pixel position (X, Y), with the
// forward deposit's wrap / zero conventions.
__device__ __forceinline__ float bilinear_p(const DevReceiver& R, float X, float Y) {
  const float xs = X - 0.5f, ys = Y - 0.5f;
  const float x0 = floorf(xs), y0 = floorf(ys);
  const float fx = xs - x0, fy = ys - y0;
  const int c0 = (int)x0, r0 = (int)y0;
  return (1 - fx) * (1 - fy) * sample_p(R, c0, r0) + fx * (1 - fy) * sample_p(R, c0 + 1, r0) +
         (1 - fx) * fy * sample_p(R, c0, r0 + 1) + fx * fy * sample_p(R, c0 + 1, r0 + 1);
}

// What the rays of one facet share: its origin and the frame of its normal
// (the slope-error perturbation's frame), as functions of the heliostat's
// parameters, and its two pool offsets.
struct FacetDual {
  Dual3 origin;
  DFrame pframe;
  int g0, g1;
};

__device__ __forceinline__ FacetDual facet_dual(const DevTask& T, const DiffTask& DT, int f) {
  float3 local, ln;
  const bool focus_flat = facet_local(T, f, local, ln);
  DFrame hf;
  hf.u = DT.u;
  hf.n = DT.fn;
  hf.v = DT.v;
  hf.identity = DT.identity != 0;
  FacetDual fd;
  fd.origin = to_world(hf, local) + d3(T.pos);
  const Dual3 fnormal = focus_flat ? to_world(hf, ln) : DT.n;
  fd.pframe = make_dframe(fnormal, false);
  fd.g0 = __ldg(T.offsets + f);
  fd.g1 = __ldg(T.offsets + (f + 1) % T.pool_size);
  return fd;
}

// Contribution of one ray (facet fd, light lab) that hit the receiver in the
// forward.
__device__ __forceinline__ void ray_adjoint(const DevTask& T, const DevReceiver& R, const FacetDual& fd, int lab,
                                            float g[K]) {
  const Dual3& origin = fd.origin;
  const float3 din = xyz(__ldg(T.samples + fd.g0 + lab));
  const float3 pert = xyz(__ldg(T.perturbations + fd.g1 + lab));
  const Dual3 np = normalize(to_world(fd.pframe, pert));
  const Dual3 in = d3(make_float3(-din.x, -din.y, -din.z));
  const Dual3 rd = normalize(in - np * (dot(np, in) * 2.0f));
  const float3 o = val(origin), d = val(rd);
  float t, u, v;
  // The receiver test with its decisions rounded as the forward's and the
  // hit point, (u, v) and distance in approximate arithmetic: the direction
  // here is the dual chain's contracted value, not the forward's, so the
  // exact position arithmetic would buy nothing.  A ray the rounding moves
  // off the receiver edge adds nothing.
  if (!receiver_hit_rx(R, o, d, t, u, v)) return;
  // energy |rd . np| eta(t) factor (receiverIntersectionUtil.cuh:17-34)
  const Dual c = dot(rd, np);
  const float sgn = c.v >= 0.0f ? 1.0f : -1.0f;
  float eta, deta;
  if (t <= 1000.0f) {
    eta = 0.99331f - 0.0001176f * t + 1.97e-8f * t * t;
    deta = -0.0001176f + 2.0f * 1.97e-8f * t;
  } else {
    eta = expf(-0.0001106f * t);
    deta = -0.0001106f * eta;
  }
  const float e = fabsf(c.v) * eta * T.factor;
  // bilinear P at the deposit position (as the forward's splat)
  const float X = v * (float)R.resolution.x, Y = u * (float)R.resolution.y;
  const float xs = X - 0.5f, ys = Y - 0.5f;
  const float x0 = floorf(xs), y0 = floorf(ys);
  const float fx = xs - x0, fy = ys - y0;
  const int c0 = (int)x0, r0 = (int)y0;
  const float p00 = sample_p(R, c0, r0), p10 = sample_p(R, c0 + 1, r0);
  const float p01 = sample_p(R, c0, r0 + 1), p11 = sample_p(R, c0 + 1, r0 + 1);
  const float pb = (1 - fx) * (1 - fy) * p00 + fx * (1 - fy) * p10 + (1 - fx) * fy * p01 + fx * fy * p11;
  const float dpx = (1 - fy) * (p10 - p00) + fy * (p11 - p01);
  const float dpy = (1 - fx) * (p01 - p00) + fx * (p11 - p10);

  float dX[K], dY[K], dt[K];
  if (R.type == 1) {
    const float3 p = make_float3(o.x + t * d.x, o.y + t * d.y, o.z + t * d.z);
    const float x = p.x - R.pos.x, z = p.z - R.pos.z;
    const float den = x * d.x + z * d.z;
    const float rr = x * x + z * z;
    const float dxz2 = d.x * d.x + d.z * d.z;
    if (!(rr > 0.0f) || !(dxz2 > 0.0f)) return;
    if (!(fabsf(den) > kGrazing * sqrtf(rr * dxz2))) {
      // Silhouette band: rays whose impact parameter b (distance of the
      // ray's horizontal line from the axis) lies within w of the radius
      // (|cos incidence| < kGrazing).  Their interior derivative grows as
      // 1/cos(incidence) and is not summed; across the band it integrates
      // to rho e v (P(silhouette) - P(inner band edge)), and the boundary
      // term of rays crossing the silhouette is -rho e v P(silhouette), so
      // together the band contributes -rho e v P(inner band edge), with
      // v = d|b|/dtheta and rho ~ (rays in the band) / w.  P is taken where
      // this ray's line would meet the cylinder with impact parameter R - w.
      const float radius = R.size.x;
      const float w = radius * (1.0f - sqrtf(1.0f - kGrazing * kGrazing));
      const Dual ox = origin.x - dc(R.pos.x), oz = origin.z - dc(R.pos.z);
      const Dual b = (ox * rd.z - oz * rd.x) * drsqrt(rd.x * rd.x + rd.z * rd.z);
      const float out = b.v >= 0.0f ? 1.0f : -1.0f;
      const float inv_dxz = rsqrtf(dxz2);
      const float hx = d.x * inv_dxz, hz = d.z * inv_dxz;  // horizontal unit direction
      const float tca = -((o.x - R.pos.x) * d.x + (o.z - R.pos.z) * d.z) / dxz2;
      const float cx = o.x + tca * d.x - R.pos.x, cz = o.z + tca * d.z - R.pos.z;  // closest approach
      const float cl = sqrtf(cx * cx + cz * cz);
      const float ux = cl > 0.0f ? cx / cl : -hz, uz = cl > 0.0f ? cz / cl : hx;
      const float back = radius * kGrazing;  // sqrt(R^2 - (R - w)^2)
      const float ex = (radius - w) * ux - back * hx, ez = (radius - w) * uz - back * hz;
      float phi = atan2f(ez, ex);
      if (phi < 0.0f) phi += kTwoPi;
      const float Xs = phi * (float)R.resolution.x / kTwoPi;
      const float ys = o.y + (tca - back * inv_dxz) * d.y;
      const float Ys = ((ys - R.pos.y) / R.size.y + 0.5f) * (float)R.resolution.y;
      const float pe = bilinear_p(R, Xs, Ys);
#pragma unroll
      for (int k = 0; k < K; ++k) g[k] -= e * pe * out * b.d[k] / w;
      return;
    }
    const float sx = (float)R.resolution.x / kTwoPi, sy = (float)R.resolution.y / R.size.y;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const float px = origin.x.d[k] + t * rd.x.d[k], py = origin.y.d[k] + t * rd.y.d[k],
                  pz = origin.z.d[k] + t * rd.z.d[k];
      dt[k] = -(x * px + z * pz) / den;
      const float qx = px + dt[k] * d.x, qy = py + dt[k] * d.y, qz = pz + dt[k] * d.z;
      dY[k] = qy * sy;
      dX[k] = (x * qz - z * qx) / rr * sx;
    }
  } else {
    const float3 N = qm::cross(R.ab, R.ac);
    const float nd = qm::dot(N, d), nn = qm::dot(N, N);
    if (!(fabsf(nd) > kGrazing * sqrtf(nn))) return;  // grazing on a plane: no boundary, detached
    const float3 abs_ = qm::mul(qm::cross(R.ac, N), 1.0f / nn), acs = qm::mul(qm::cross(N, R.ab), 1.0f / nn);
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const float3 dox = make_float3(origin.x.d[k], origin.y.d[k], origin.z.d[k]);
      const float3 ddx = make_float3(rd.x.d[k], rd.y.d[k], rd.z.d[k]);
      dt[k] = -(qm::dot(N, dox) + t * qm::dot(N, ddx)) / nd;
      const float3 q = make_float3(dox.x + t * ddx.x + dt[k] * d.x, dox.y + t * ddx.y + dt[k] * d.y,
                                   dox.z + t * ddx.z + dt[k] * d.z);
      dY[k] = qm::dot(q, abs_) * (float)R.resolution.y;
      dX[k] = qm::dot(q, acs) * (float)R.resolution.x;
    }
  }
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const float de = (sgn * c.d[k] * eta + fabsf(c.v) * deta * dt[k]) * T.factor;
    g[k] += e * (dpx * dX[k] + dpy * dY[k]) + pb * de;
  }
  // Image edges (rows of both receivers, columns of a rectangle): rays within
  // kEdgeBand pixels of an edge estimate the boundary term -rho e P
  // (outward pixel velocity) of rays leaving or entering across it, with P
  // taken on the edge itself (half of an edge deposit falls outside).
  const float by = kEdgeBand;
  const float H = (float)R.resolution.y, W = (float)R.resolution.x;
  if (Y < by) {
    const float pe = bilinear_p(R, X, 0.0f);
    for (int k = 0; k < K; ++k) g[k] += e * pe * dY[k] / by;
  }
  if (H - Y < by) {
    const float pe = bilinear_p(R, X, H);
    for (int k = 0; k < K; ++k) g[k] -= e * pe * dY[k] / by;
  }
  if (R.type == 0) {
    if (X < by) {
      const float pe = bilinear_p(R, 0.0f, Y);
      for (int k = 0; k < K; ++k) g[k] += e * pe * dX[k] / by;
    }
    if (W - X < by) {
      const float pe = bilinear_p(R, W, Y);
      for (int k = 0; k < K; ++k) g[k] -= e * pe * dX[k] / by;
    }
  }
}


// Facet window of the adjoint, per warp (as the trace kernel's): the
// FacetDual of 32 consecutive facets, one per lane, stored component-major so
// that lanes reading different slots touch different banks.
#ifndef QM_BWD_THREADS
#define QM_BWD_THREADS 32
#endif
#ifndef QM_BWD_MIN_BLOCKS
#define QM_BWD_MIN_BLOCKS 20
#endif
constexpr int kBwdThreads = QM_BWD_THREADS;
constexpr int kDual3Words = 3 * (1 + K);
struct AdjointWindow {
  float origin[kDual3Words][kBwdThreads];
  float frame[3 * kDual3Words][kBwdThreads];  // u, n, v
  int g0[kBwdThreads], g1[kBwdThreads], identity[kBwdThreads];
};

__device__ __forceinline__ void put_dual3(float (*dst)[kBwdThreads], int slot, const Dual3& a) {
  const Dual* c[3] = {&a.x, &a.y, &a.z};
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    dst[i * (1 + K)][slot] = c[i]->v;
#pragma unroll
    for (int k = 0; k < K; ++k) dst[i * (1 + K) + 1 + k][slot] = c[i]->d[k];
  }
}

__device__ __forceinline__ Dual3 get_dual3(const float (*src)[kBwdThreads], int slot) {
  Dual3 a;
  Dual* c[3] = {&a.x, &a.y, &a.z};
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    c[i]->v = src[i * (1 + K)][slot];
#pragma unroll
    for (int k = 0; k < K; ++k) c[i]->d[k] = src[i * (1 + K) + 1 + k][slot];
  }
  return a;
}

__global__ void __launch_bounds__(kBwdThreads, QM_BWD_MIN_BLOCKS) diff_backward_kernel(BackwardParams p) {
  __shared__ AdjointWindow win;
  const int lane = threadIdx.x & 31;
  const int wbase = threadIdx.x & ~31;
  const long long warp = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const long long chunk = p.chunk_begin + warp;
  if (chunk >= p.total_chunks) return;
  const int nl = p.light_end - p.light_begin;
  const int t = find_task(p.chunk_prefix, p.num_tasks, chunk);
  const int r0 = (int)(chunk - __ldg(p.chunk_prefix + t)) * kChunk;
  const DevTask& T = p.tasks[t];
  const DiffTask& DT = p.dtasks[t];
  const DevReceiver& R = p.receivers[T.receiver];
  const int r_end = T.num_facets * nl;
  const int iters = min(kChunkIters, (r_end - r0 + 31) >> 5);
  int f = (r0 + lane) / nl;
  int l = (r0 + lane) - f * nl;
  float g[K];
#pragma unroll
  for (int k = 0; k < K; ++k) g[k] = 0.0f;
  int base = 0;
  bool filled = false;  // warp-uniform
  for (int it = 0; it < iters; ++it) {
    const bool active = r0 + it * 32 + lane < r_end;
    const unsigned bits = __ldg(p.hit_bits + warp * kChunkIters + it);
    // The facets of an iteration lie within 32 of lane 0's (see the trace
    // kernel); refill the window when a lane with a hit needs one past it.
    const int f0 = __shfl_sync(0xffffffffu, f, 0);
    const bool hit = active && ((bits >> lane) & 1u);
    if (__any_sync(0xffffffffu, hit && (!filled || f - base >= 32))) {
      __syncwarp();
      base = f0;
      filled = true;
      const int fw = base + lane;
      if (fw < T.num_facets) {
        const FacetDual fd = facet_dual(T, DT, fw);
        const int slot = wbase + lane;
        put_dual3(win.origin, slot, fd.origin);
        put_dual3(win.frame, slot, fd.pframe.u);
        put_dual3(win.frame + kDual3Words, slot, fd.pframe.n);
        put_dual3(win.frame + 2 * kDual3Words, slot, fd.pframe.v);
        win.g0[slot] = fd.g0;
        win.g1[slot] = fd.g1;
        win.identity[slot] = fd.pframe.identity ? 1 : 0;
      }
      __syncwarp();
    }
    if (hit) {
      const int slot = wbase + (f - base);
      FacetDual fd;
      fd.origin = get_dual3(win.origin, slot);
      fd.pframe.u = get_dual3(win.frame, slot);
      fd.pframe.n = get_dual3(win.frame + kDual3Words, slot);
      fd.pframe.v = get_dual3(win.frame + 2 * kDual3Words, slot);
      fd.pframe.identity = win.identity[slot] != 0;
      fd.g0 = win.g0[slot];
      fd.g1 = win.g1[slot];
      ray_adjoint(T, R, fd, p.light_begin + l, g);
    }
    f += p.lights_q32;
    l += p.lights_r32;
    if (l >= nl) {
      l -= nl;
      ++f;
    }
  }
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double s = g[k];
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if (lane == 0 && s != 0.0) atomicAdd(p.grad + (size_t)T.power_slot * K + k, s);
  }
}

// ---- smoothing and loss ---------------------------------------------------------
__global__ void gauss_rows_kernel(const float* in, float* out, int w, int h, const float* wt, int radius, bool wrap) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= w || y >= h) return;
  float s = 0.0f;
  for (int k = -radius; k <= radius; ++k) {
    int c = x + k;
    if (wrap) c = ((c % w) + w) % w;
    if (c < 0 || c >= w) continue;
    s += wt[k < 0 ? -k : k] * in[(size_t)y * w + c];
  }
  out[(size_t)y * w + x] = s;
}

__global__ void gauss_cols_kernel(const float* in, float* out, int w, int h, const float* wt, int radius) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= w || y >= h) return;
  float s = 0.0f;
  for (int k = -radius; k <= radius; ++k) {
    const int r = y + k;
    if (r < 0 || r >= h) continue;
    s += wt[k < 0 ? -k : k] * in[(size_t)r * w + x];
  }
  out[(size_t)y * w + x] = s;
}

__global__ void round_kernel(const double* in, float* out, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (float)in[i];
}

__global__ void loss_kernel(const float* flux, const float* target, float* resid, long long n, double* loss) {
  __shared__ double part[8];
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double s = 0.0;
  if (i < n) {
    const float diff = flux[i] - target[i];
    resid[i] = 2.0f * diff;
    s = (double)diff * diff;
  }
  for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) b += part[k];
    if (b != 0.0) atomicAdd(loss, b);
  }
}

}  // namespace

cudaError_t launch_diff_prep(const PrepItem* items, int n, const DevTask* tasks, DiffTask* out, cudaStream_t stream) {
  if (n <= 0) return cudaSuccess;
  diff_prep_kernel<<<(n + 127) / 128, 128, 0, stream>>>(items, n, tasks, out);
  return cudaGetLastError();
}

cudaError_t launch_diff_backward(const BackwardParams& params, cudaStream_t stream) {
  const long long nl = params.light_end - params.light_begin;
  if (params.chunk_begin < 0) return cudaErrorInvalidValue;
  if (nl <= 0 || params.total_chunks <= params.chunk_begin) return cudaSuccess;
  BackwardParams p = params;
  p.lights_q32 = (int)(32 / nl);
  p.lights_r32 = (int)(32 % nl);
  const long long warps_per_block = kBwdThreads / 32;
  const long long blocks = (p.total_chunks - p.chunk_begin + warps_per_block - 1) / warps_per_block;
  if (blocks > 0x7fffffffLL) return cudaErrorInvalidValue;
  diff_backward_kernel<<<(unsigned)blocks, kBwdThreads, 0, stream>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_gauss(const float* in, float* tmp, float* out, int width, int height, const float* weights,
                         int radius, bool wrap_cols, cudaStream_t stream) {
  if (width <= 0 || height <= 0) return cudaSuccess;
  const dim3 grid((width + 127) / 128, height);
  gauss_rows_kernel<<<grid, 128, 0, stream>>>(in, tmp, width, height, weights, radius, wrap_cols);
  gauss_cols_kernel<<<grid, 128, 0, stream>>>(tmp, out, width, height, weights, radius);
  return cudaGetLastError();
}

cudaError_t launch_round_deposit(const double* in, float* out, long long n, cudaStream_t stream) {
  if (n <= 0) return cudaSuccess;
  round_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(in, out, n);
  return cudaGetLastError();
}

cudaError_t launch_loss(const float* flux, const float* target, float* resid, long long n, double* loss,
                        cudaStream_t stream) {
  if (n <= 0) return cudaSuccess;
  loss_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(flux, target, resid, n, loss);
  return cudaGetLastError();
}

}  // namespace qm
