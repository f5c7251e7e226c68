// Device-side per-sun preparation (prep.cu).
#pragma once

#include <cuda_runtime.h>

#include "device_scene.h"

namespace qm {

// One (sun, heliostat) to prepare.  The task already holds the heliostat's
// sun-independent fields; the kernel fills its normal and facet frame and
// writes the heliostat's sub-heliostat parallelograms and traversal record
// into the sun's grid arrays.
struct PrepItem {
  int task;         // index into the task array
  int num_sub;      // sub-heliostats of the heliostat
  int sub_first;    // grid-local id of its first sub-heliostat
  float3 focus;     // aim point (sun-independent)
  float3 sun_dir;   // direction of travel of the sun's rays
  // Differentiable parameters (zero for plain batches): the aim point moves
  // by aim_offset.x * aim_u + aim_offset.y * aim_v; the normal then turns by
  // normal_offset (radians) about the u and v axes of its own frame.
  float2 aim_offset, normal_offset;
  float3 aim_u, aim_v;
  // Shadow-free test (qm::shadow_free): sun axis and world-space tangent of
  // the largest sun-shape angle (< 0: unbounded, never shadow-free).
  float3 shadow_axis;
  float shadow_tan;
  // Block-free test (qm::block_free): theta_sun + 2 theta_slope (< 0: never),
  // and where the heliostat's per-sub-heliostat flags go.
  float block_theta;
  int* sub_free;
  int* sub_cand;  // kMaxCandidates per sub-heliostat
  float4* sub_frames;  // 6 per sub-heliostat (DevGrid::sub_frames)
  float3* verts;    // out: 3 float3 (B, A, C) per sub-heliostat
  float4* subv;     // out: 3 float4 per sub-heliostat (A, B - A, C - A)
  float4* bound;    // out: 5 float4 traversal record
  int4* hsub;       // out: (first, count, lattice rows, lattice columns)
};

struct PoolRotation {
  const float4* in;  // local sun-shape pool, n entries
  float4* out;       // world-space tracer copy, n_out = n + L entries (entry i = pool entry i % n)
  int n, n_out;
  SunFrame sun;
};

// Walk-free flags of a plain scene: shadow flags per task into shadow_out,
// block flags per sub-heliostat into each grid's sub_free array.
struct WalkFlagParams {
  const DevTask* tasks;
  int n;
  const DevGrid* grids;
  float3 sun_axis;  // toward the sun
  float sun_tan;    // tan of the largest sun-shape angle (< 0: unbounded)
  float3 sun_dir;   // direction of travel
  float block_theta;
  int* shadow_out;       // per task: DevTask::shadow_free code
  int* shadow_cand_out;  // per task: kMaxCandidates DevTask::shadow_cand entries
  int max_sub;           // most sub-heliostats of any task
};
cudaError_t launch_walk_flags(const WalkFlagParams& p, cudaStream_t stream);

cudaError_t launch_prep(const PrepItem* items, int n, DevTask* tasks, cudaStream_t stream);
// Shadow-free flags of the prepared tasks; grids: the tasks' grids with their
// prepared traversal records.  Run after launch_prep.
// max_sub: the most sub-heliostats of any item (one thread per heliostat and
// per sub-heliostat).
cudaError_t launch_shadow_flags(const PrepItem* items, int n, int max_sub, DevTask* tasks, const DevGrid* grids,
                                cudaStream_t stream);
// max_out: the largest n_out of the jobs.
cudaError_t launch_rotate_pools(const PoolRotation* jobs, int n_jobs, int max_out, cudaStream_t stream);

}  // namespace qm
