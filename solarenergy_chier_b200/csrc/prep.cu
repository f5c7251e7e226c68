// Per-sun scene preparation on the device: for every (sun, heliostat) of a
// batch, the sun-dependent half of SceneProcessor::processScene
// (Scene/SceneProcessor.cpp:22-39): the heliostat normal
// (Heliostat::CSetNormal, Heliostat.cu:15-20), its corner / sub-heliostat
// parallelograms (Heliostat::CSetWorldVertex, Heliostat.cu:22-40;
// FocusFlatRectangleHelio::CGetSubHeliostatVertexes, FocusFlatRectangleHelio.cu:123-227),
// the traversal record and the tracer's facet frame; and the world-space
// sun-shape pool of every sun.
//
// The arithmetic is helio_geom.h's, shared with the host scene code; this
// unit is compiled with -fmad=false, so a heliostat prepared here equals the
// host's bit for bit.
#include "prep.h"

#include "helio_geom.h"
#include "ray_geom.h"
#include "shadow.h"

namespace qm {
namespace {

__global__ void prep_kernel(const PrepItem* items, int n, DevTask* tasks) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const PrepItem it = items[i];
  DevTask& T = tasks[it.task];
  float3 aim = it.focus;
  if (it.aim_offset.x != 0.0f || it.aim_offset.y != 0.0f)
    aim = qs::add(qs::add(aim, qs::mul(it.aim_u, it.aim_offset.x)), qs::mul(it.aim_v, it.aim_offset.y));
  float3 normal = helio_normal(T.pos, aim, it.sun_dir);
  if (it.normal_offset.x != 0.0f || it.normal_offset.y != 0.0f) {
    const Frame f0 = qs::make_frame(normal, false);
    normal = qs::normalize(
        qs::add(qs::add(normal, qs::mul(f0.u, it.normal_offset.x)), qs::mul(f0.v, it.normal_offset.y)));
  }
  T.normal = normal;
  const Frame hf = qs::make_frame(normal, T.type == 1);
  T.fu = hf.u;
  T.fn = hf.n;
  T.fv = hf.v;
  T.frame_identity = hf.identity ? 1 : 0;
  float3* v = it.verts;
  if (T.type == 0) {
    float3 c[4];
    flat_vertices(T.size, normal, T.pos, c);
    v[0] = c[0];
    v[1] = c[1];
    v[2] = c[2];
  } else {
    const float2 len = sub_lengths(T.size, T.gap, T.row_col);
    for (int s = 0; s < it.num_sub; ++s)
      focus_flat_sub_vertices(len, T.local_centers[s], T.local_normals[s], normal, T.pos, v + 3 * s);
  }
  for (int s = 0; s < it.num_sub; ++s) {
    const float3 B = v[3 * s], A = v[3 * s + 1], C = v[3 * s + 2];
    const float3 ab = qs::sub(B, A), ac = qs::sub(C, A);
    it.subv[3 * s] = make_float4(A.x, A.y, A.z, ab.x);
    it.subv[3 * s + 1] = make_float4(ab.y, ab.z, ac.x, ac.y);
    it.subv[3 * s + 2] = make_float4(ac.z, 0.f, 0.f, 0.f);
  }
  int2 rc;
  heliostat_record(v, it.num_sub, T.row_col, T.pos, normal, it.bound, &rc);
  *it.hsub = make_int4(it.sub_first, it.num_sub, rc.x, rc.y);
}

// DevGrid::sub_free code of a block_candidates result: 1 nothing to hit,
// k + 1 for k listed candidates, 0 walk (too many, or not enumerable).
__device__ __forceinline__ int candidate_code(int k) {
  return k == 0 ? 1 : (k > 0 && k <= kMaxCandidates ? k + 1 : 0);
}

// Walk codes of the prepared tasks: thread j handles task j / (1 + max_sub),
// slot j % (1 + max_sub): slot 0 its shadow walks, slot 1 + s the block
// walks of its sub-heliostat s (each a capsule enumeration of its own).
__global__ void shadow_kernel(const PrepItem* items, int n, int max_sub, DevTask* tasks, const DevGrid* grids) {
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int i = (int)(j / (1 + max_sub)), slot = (int)(j % (1 + max_sub));
  if (i >= n) return;
  const PrepItem& it = items[i];
  DevTask& T = tasks[it.task];
  const DevGrid& G = grids[T.grid];
  const ShadowGrid view{G.pos, G.interval, G.cells, G.bound, G.cell_range, G.entries};
  if (slot == 0) {
    T.shadow_free = candidate_code(it.shadow_tan >= 0.0f ? shadow_candidates(view, T.own, it.shadow_axis,
                                                                            it.shadow_tan, T.shadow_cand,
                                                                            kMaxCandidates)
                                                         : -1);
    return;
  }
  const int s = slot - 1;
  if (s >= it.num_sub) return;
  Frame hf;
  hf.u = T.fu;
  hf.n = T.fn;
  hf.v = T.fv;
  hf.identity = T.frame_identity != 0;
  const float3 nrm = T.type == 1 ? qs::to_world(hf, T.local_normals[s]) : T.normal;
  sub_frames(T, s, it.sub_frames + 6 * s);
  const int k = it.block_theta >= 0.0f ? block_candidates(view, T.own, it.verts + 3 * s, it.sun_dir, nrm,
                                                         it.block_theta, it.sub_cand + kMaxCandidates * s,
                                                         kMaxCandidates)
                                       : -1;
  it.sub_free[s] = candidate_code(k);
}

// Walk codes of a plain scene's heliostats (its task templates), with the
// same thread layout as shadow_kernel; the sub-heliostat parallelograms are
// read back from the traversal form (A, B - A, C - A) -- the tests are
// conservative far above that rounding.
__global__ void walk_flags_kernel(WalkFlagParams p) {
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int i = (int)(j / (1 + p.max_sub)), slot = (int)(j % (1 + p.max_sub));
  if (i >= p.n) return;
  const DevTask& T = p.tasks[i];
  const DevGrid& G = p.grids[T.grid];
  const ShadowGrid view{G.pos, G.interval, G.cells, G.bound, G.cell_range, G.entries};
  if (slot == 0) {
    p.shadow_out[i] = candidate_code(p.sun_tan >= 0.0f ? shadow_candidates(view, T.own, p.sun_axis, p.sun_tan,
                                                                           p.shadow_cand_out + kMaxCandidates * i,
                                                                           kMaxCandidates)
                                                        : -1);
    return;
  }
  const int s = slot - 1;
  const int4 hs = G.hsub[T.own];
  if (s >= hs.y) return;
  Frame hf;
  hf.u = T.fu;
  hf.n = T.fn;
  hf.v = T.fv;
  hf.identity = T.frame_identity != 0;
  int* sub_free = const_cast<int*>(G.sub_free);
  int* sub_cand = const_cast<int*>(G.sub_cand);
  sub_frames(T, s, const_cast<float4*>(G.sub_frames) + 6 * (hs.x + s));
  const float4* q = G.subv + 3 * (hs.x + s);
  const float3 A = make_float3(q[0].x, q[0].y, q[0].z);
  const float3 bac[3] = {make_float3(A.x + q[0].w, A.y + q[1].x, A.z + q[1].y), A,
                         make_float3(A.x + q[1].z, A.y + q[1].w, A.z + q[2].x)};
  const float3 nrm = T.type == 1 ? qs::to_world(hf, T.local_normals[s]) : T.normal;
  const int k = p.block_theta >= 0.0f ? block_candidates(view, T.own, bac, p.sun_dir, nrm, p.block_theta,
                                                        sub_cand + kMaxCandidates * (hs.x + s), kMaxCandidates)
                                      : -1;
  sub_free[hs.x + s] = candidate_code(k);
}

// Pool of instance blockIdx.y turned by that instance's sun frame.
__global__ void rotate_pools_kernel(const PoolRotation* jobs) {
  const PoolRotation J = jobs[blockIdx.y];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= J.n_out) return;
  const int k = i % J.n;
  float3 d = make_float3(J.in[k].x, J.in[k].y, J.in[k].z);
  if (!J.sun.identity) {
    Frame f;
    f.u = J.sun.u;
    f.n = J.sun.n;
    f.v = J.sun.v;
    f.identity = false;
    d = qs::to_world(f, d);
  }
  J.out[i] = make_float4(d.x, d.y, d.z, 0.0f);
}

}  // namespace

cudaError_t launch_prep(const PrepItem* items, int n, DevTask* tasks, cudaStream_t stream) {
  if (n <= 0) return cudaSuccess;
  prep_kernel<<<(n + 127) / 128, 128, 0, stream>>>(items, n, tasks);
  return cudaGetLastError();
}

cudaError_t launch_shadow_flags(const PrepItem* items, int n, int max_sub, DevTask* tasks, const DevGrid* grids,
                                cudaStream_t stream) {
  if (n <= 0) return cudaSuccess;
  if (max_sub < 0) return cudaErrorInvalidValue;
  const long long threads = (long long)n * (1 + max_sub);
  shadow_kernel<<<(unsigned)((threads + 63) / 64), 64, 0, stream>>>(items, n, max_sub, tasks, grids);
  return cudaGetLastError();
}

cudaError_t launch_walk_flags(const WalkFlagParams& p, cudaStream_t stream) {
  if (p.n <= 0) return cudaSuccess;
  if (p.max_sub < 0) return cudaErrorInvalidValue;
  const long long threads = (long long)p.n * (1 + p.max_sub);
  walk_flags_kernel<<<(unsigned)((threads + 63) / 64), 64, 0, stream>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_rotate_pools(const PoolRotation* jobs, int n_jobs, int max_out, cudaStream_t stream) {
  if (n_jobs <= 0 || max_out <= 0) return cudaSuccess;
  if (n_jobs > 65535) return cudaErrorInvalidValue;
  rotate_pools_kernel<<<dim3((max_out + 255) / 256, n_jobs), 256, 0, stream>>>(jobs);
  return cudaGetLastError();
}

}  // namespace qm
