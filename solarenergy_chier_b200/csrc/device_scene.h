// Plain-old-data views of a processed scene, as the sm_100a kernels read them.
// Built on the host by capi.cpp from the float32 scene model (scene.h).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace qm {

// One RectangleGrid (Scene/DataStructure/Grid/RectangleGrid.cuh:13-52) in
// traversal form.
// Candidate heliostats kept per sub-heliostat (DevGrid::sub_cand) and per
// task (DevTask::shadow_cand) for the walk pre-tests.
constexpr int kMaxCandidates = 6;

struct DevGrid {
  float3 pos;
  float3 interval;
  int3 cells;
  int max_steps;        // DDA step bound: cells.x + cells.y + cells.z + 2
  const int2* cell_range;  // [begin, end) of each cell's entries
  const int4* entries;     // per cell entry: grid-local heliostat id, first sub-heliostat, count, 0
  const float4* bound;  // 5 float4 per grid-local heliostat: (centre, window margin), (axis_k, half extent_k)
                        // for k = lattice x, normal, lattice z, then (x0, 1/px, z0, 1/pz)
  const int4* hsub;     // (first sub-heliostat id, count, lattice rows, lattice columns) per grid-local heliostat
  const float4* subv;   // 3 float4 per sub-heliostat: A.xyz AB.x | AB.yz AC.xy | AC.z
  // Per sub-heliostat, for its facets' block walks (qm::block_candidates):
  // 1 = skipped (nothing can be hit), k + 1 = only the k <= kMaxCandidates
  // heliostats in sub_cand[kMaxCandidates * sub ...] can be hit (a ray
  // meeting none of their padded boxes skips the walk), 0 = walk.
  const int* sub_free;
  const int* sub_cand;
  // Per sub-heliostat, for the tracer's facet window: the frame of its
  // facets' world normal (u, n, v; identity flag in u.w) and, for focus-flat
  // heliostats, the flipped frame of its local normal that places its facets
  // (same layout): 6 float4, written with the walk codes for the current sun.
  const float4* sub_frames;
};

struct DevReceiver {
  int type;             // 0 rectangle, 1 cylinder
  int2 resolution;      // x = columns, y = rows
  float* image;         // resolution.x * resolution.y floats, row-major by row
  double* deposit;      // bilinear-deposit launches: FP64 accumulator of the same shape (else unused)
  float3 a, ab, ac;     // rectangle: vertex 0, v1 - v0, v3 - v0
  float3 pos, size;     // cylinder: centre, (radius, height, -)
  float rcp_height;     // cylinder: 1 / height rounded to nearest (host division)
};

// One heliostat to trace (a HeliostatArgument plus the per-heliostat
// constants of QuasiMonteCarloRayTracer::rayTracing).
struct DevTask {
  int type;             // 0 flat, 1 focus-flat
  int grid;
  int receiver;
  int own;              // grid-local heliostat id, skipped by the DDA
  int num_facets;
  int power_slot;
  int2 row_col;
  int2 sub_row_col;
  float pixel_length;
  float factor;
  float2 gap;
  float2 sub_length;    // x along z (rows), y along x (columns)
  float3 size;
  float3 pos;
  float3 normal;
  float3 fu, fn, fv;    // frame of the heliostat normal (plain or flipped variant)
  int frame_identity;
  const float3* local_centers;  // focus-flat: per sub-heliostat
  const float3* local_normals;
  const int* offsets;   // num_facets + 1 pool offsets
  const float4* samples;        // sun-shape pool already turned into world space by this task's sun
  const float4* perturbations;  // slope-error pool (local frame of the facet normal)
  int pool_size;                // P = groups x lights per group
  // Shadow walks of this heliostat's rays (qm::cone_candidates around the
  // sun-shape cone): 1 = skipped (nothing can shadow them), k + 1 = only the
  // k listed heliostats can (a ray meeting none of their padded boxes skips
  // its walk), 0 = walk.
  int shadow_free;
  int shadow_cand[kMaxCandidates];
};

struct SunFrame {
  float3 u, n, v;
  int identity;
};

// Per-ray outcome codes written by the hit-record variant; a hit stores its
// pixel index (>= 0).
enum RayCode : int32_t { kShadowed = -1, kBlocked = -2, kMissed = -3, kNotTraced = -4 };

// Diagnostic counters (unsigned long long each).
enum DiagSlot { kDiagClamped = 0, kDiagDdaCap = 1, kDiagSlots = 4 };

// Warp chunk: every launch over tasks hands each warp kChunkIters x 32
// consecutive rays of one task (trace_kernel, diff_backward_kernel; hit bits
// are one word per chunk iteration).  Larger chunks amortise the per-chunk
// work (task lookup, facet window fill, power reduction) over more rays.
#ifndef QM_CHUNK_ITERS
#define QM_CHUNK_ITERS 64
#endif
constexpr int kChunkIters = QM_CHUNK_ITERS;
constexpr int kChunk = 32 * kChunkIters;

struct TraceParams {
  const DevGrid* grids;
  const DevReceiver* receivers;
  const DevTask* tasks;
  const long long* facet_prefix;  // num_tasks + 1 prefix sums of warp chunks per task
  int num_tasks;
  long long total_facets;         // end of the launch's warp chunks (chunks [chunk_begin, total_facets))
  long long chunk_begin;          // first warp chunk of the launch (0: all)
  int light_begin, light_end;     // light indexes traced per facet
  int lights_q32, lights_r32;     // 32 / (light_end - light_begin) and 32 % it (set by the launcher)
  double* power;                  // FP64 per-slot power accumulators
  // flux and bilinear-deposit launches: when set, each warp chunk writes its
  // rays' FP64 energy sum to chunk_power[chunk - chunk_begin] and
  // launch_power_reduce (power.cu) adds them per task into power, in a fixed
  // order with compensation; when NULL, one double atomic per chunk
  double* chunk_power;
  unsigned long long* diag;
  // bilinear-deposit and hit-bit variants: one word per warp iteration of the
  // launch (chunk - chunk_begin), bit i = lane i's ray hit the receiver; may
  // be NULL for the bilinear deposit
  uint32_t* hit_bits;
  // hit-record variant only
  int32_t* records;
  int record_task;
  int record_facet_begin, record_facet_end;
};

}  // namespace qm
