// Sample pools and per-facet pool offsets, generated on the device.
//
// The reference draws both pools from cuRAND XORWOW seeded with time(NULL)
// (Scene/SceneProcessor.cu:147-271, Tool/RandomNumberGenerator/).  Here they
// come from the scrambled Sobol streams of sampling.h, so a seed reproduces
// a pool exactly; the mapping from uniforms to directions follows the
// reference.
#include "pools.h"
#include "sampling.h"
#include "vecmath.h"

namespace qm {
namespace {

// samplelights::max_less_index (Scene/SceneProcessor.cu:46-59).
__device__ __forceinline__ int max_less_index(const float2* cdf, float value, int n) {
  int left = 0, right = n;
  while (left <= right) {
    int mid = (left + right) >> 1;
    float y = cdf[mid].y;
    if (value > y)
      left = mid + 1;
    else if (value < y)
      right = mid - 1;
    else
      return mid;
  }
  return right;
}

// samplelights::linear_interpolation (Scene/SceneProcessor.cu:61-81): the
// reference's Buie inverse CDF, including its arctangent warp of the core
// and its tail formula that lands at >= 9.3 mrad.
__device__ __forceinline__ float buie_theta(float uniform, const BuieTable& b) {
  float u = uniform * b.A;
  if (u < b.less_465) {
    int id = max_less_index(b.cdf, u, b.n);
    u = (u - b.cdf[id].y) * b.k[id] + b.cdf[id].x;
    u = atanf(sqrtf(u / 4.65f) * 0.5016916f);
  } else {
    u = powf((u - b.less_465) * b.B + b.C, 1 / (b.gamma + 1));
    float ri2 = 0.5016916f * 0.5016916f;
    float ro2 = 1.340874f * 1.340874f;
    u = atanf(sqrtf(ro2 + (u - 4.65f) / 4.65f * (ro2 - ri2)));
  }
  return u / 100.0f;
}

__global__ void pool_kernel(PoolParams p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.pool_size) return;
  uint32_t a, b;
  sobol2_owen((uint32_t)i, p.seed_sun, a, b);
  float3 s;
  if (p.sunshape == kSunshapePillbox) {
    // Uniform over the disc of half-angle h: cos(theta) uniform in [cos h, 1].
    double th = 2.0 * asin(sqrt(unit_open(a)) * sin(0.5 * (double)p.half_angle));
    double ph = 2.0 * M_PI * unit_open(b);
    s = make_float3((float)(sin(th) * cos(ph)), (float)cos(th), (float)(sin(th) * sin(ph)));
  } else {
    // samplelights::map_angle2xyz (Scene/SceneProcessor.cu:95-103) with the
    // reference's float constants.
    float theta = buie_theta(unit_float(a), p.buie);
    float phi = unit_float(b) * 2 * 3.141592654f;
    s = make_float3(sinf(theta) * cosf(phi), cosf(theta), sinf(theta) * sinf(phi));
  }
  p.samples[i] = make_float4(s.x, s.y, s.z, 0.0f);

  // Slope error: samplelights::map_permuation (Scene/SceneProcessor.cu:83-93),
  // normalize(N(0, sigma), 1, N(0, sigma)), Gaussians by Box-Muller.
  sobol2_owen((uint32_t)i, p.seed_slope, a, b);
  double r = sqrt(-2.0 * log(unit_open(a)));
  double w = 2.0 * M_PI * unit_open(b);
  float3 d = make_float3((float)((double)p.sigma * r * cos(w)), 1.0f, (float)((double)p.sigma * r * sin(w)));
  d = normalize(d);
  p.perturbations[i] = make_float4(d.x, d.y, d.z, 0.0f);
}

__global__ void offsets_kernel(int* out, long long count, uint32_t seed, int heliostat, int pool) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  out[i] = facet_offset(seed, (uint32_t)heliostat, (uint32_t)i, (uint32_t)pool);
}

__global__ void xyz_to_float4_kernel(const float* xyz, float4* out, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = make_float4(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], 0.0f);
}

}  // namespace

cudaError_t launch_pool(const PoolParams& p, cudaStream_t stream) {
  if (p.pool_size <= 0) return cudaSuccess;
  pool_kernel<<<(p.pool_size + 255) / 256, 256, 0, stream>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_offsets(int* out, long long count, uint32_t seed, int heliostat, int pool, cudaStream_t stream) {
  if (count <= 0) return cudaSuccess;
  offsets_kernel<<<(unsigned)((count + 255) / 256), 256, 0, stream>>>(out, count, seed, heliostat, pool);
  return cudaGetLastError();
}

cudaError_t launch_xyz_to_float4(const float* xyz, float4* out, int n, cudaStream_t stream) {
  if (n <= 0) return cudaSuccess;
  xyz_to_float4_kernel<<<(n + 255) / 256, 256, 0, stream>>>(xyz, out, n);
  return cudaGetLastError();
}

}  // namespace qm
