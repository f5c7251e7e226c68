// Sample-pool and facet-offset generation (device) and the Buie sun-shape
// table (host).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

namespace qm {

enum Sunshape : int { kSunshapeBuie = 0, kSunshapePillbox = 1 };

// Device view of the reference's Buie inverse-CDF table.
struct BuieTable {
  const float2* cdf;  // n + 1 (theta mrad, cumulative) pairs
  const float* k;     // n slopes
  int n;
  float less_465;     // integral of the core, 0..4.65 mrad
  float gamma, A, B, C;
};

// Host copy: SceneProcessor::set_samplelights parameters
// (Scene/SceneProcessor.cu:196-240 with parameters_generate, :23-44), float
// arithmetic in the reference's order.
struct BuieHost {
  std::vector<float2> cdf;
  std::vector<float> k;
  float less_465 = 0.f, gamma = 0.f, A = 0.f, B = 0.f, C = 0.f, kappa = 0.f;
};
BuieHost build_buie_table(float csr, int num_group);

struct PoolParams {
  float4* samples;
  float4* perturbations;
  int pool_size;
  int sunshape;
  float half_angle;   // pillbox half-angle, radians
  float sigma;        // slope-error standard deviation, radians
  uint32_t seed_sun;
  uint32_t seed_slope;
  BuieTable buie;
};

cudaError_t launch_pool(const PoolParams& p, cudaStream_t stream);
cudaError_t launch_offsets(int* out, long long count, uint32_t seed, int heliostat, int pool, cudaStream_t stream);
cudaError_t launch_xyz_to_float4(const float* xyz, float4* out, int n, cudaStream_t stream);
// Adds to *bad the number of the n xyz vectors whose squared length is outside
// [0.25, 4] or NaN.
cudaError_t launch_count_non_unit(const float* xyz, int n, unsigned* bad, cudaStream_t stream);
// *out (zeroed by the caller) = bits of the largest tan(angle from +y) over
// the pool (+inf if some direction has y <= 0).
cudaError_t launch_pool_tan(const float4* pool, int n, unsigned* out, cudaStream_t stream);
// Offsets of all heliostats; seg (device) holds heliostats + 1 segment starts.
cudaError_t launch_offsets_all(int* out, const long long* seg, int heliostats, long long total, uint32_t seed, int pool,
                               cudaStream_t stream);
struct SunFrame;
// Tracer copies of the pools (n_out = P + L entries, entry i = pool entry
// i % P; samples turned into world space by the sun frame).
cudaError_t launch_trace_pools(const float4* samples, const float4* perturbations, int n, int n_out,
                               const SunFrame& sun, float4* out, float4* pert_out, cudaStream_t stream);

}  // namespace qm
