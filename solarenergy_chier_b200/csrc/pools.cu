// Sample pools and per-facet pool offsets, generated on the device.
//
// The reference draws both pools from cuRAND XORWOW seeded with time(NULL)
// (Scene/SceneProcessor.cu:147-271, Tool/RandomNumberGenerator/).  Here they
// come from the scrambled Sobol streams of sampling.h, so a seed reproduces
// a pool exactly; the mapping from uniforms to directions follows the
// reference.
#include "pools.h"
#include "device_scene.h"
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

// Facet offsets of every heliostat in one launch: element i of the buffer
// belongs to heliostat h with seg[h] <= i < seg[h + 1].
__global__ void offsets_all_kernel(int* out, const long long* seg, int heliostats, uint32_t seed, int pool) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= seg[heliostats]) return;
  int lo = 0, hi = heliostats - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (seg[mid] <= i) lo = mid; else hi = mid - 1;
  }
  out[i] = facet_offset(seed, (uint32_t)lo, (uint32_t)(i - seg[lo]), (uint32_t)pool);
}

// The pools as the tracer reads them: n_out = P + L entries, entry i holding
// pool entry i % P, so that offset + light index never wraps; sun-shape
// samples turned into world space by the sun frame, exactly as the reference
// turns each one per ray (local2world_rotate of the sample about
// -sun_direction, RectangleReceiverRectangleGridRayTracing.cu:16).
__global__ void trace_pools_kernel(const float4* in, const float4* pert, int n, int n_out, SunFrame sun, float4* out,
                                   float4* pert_out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_out) return;
  const int k = i % n;
  pert_out[i] = pert[k];
  float3 d = make_float3(in[k].x, in[k].y, in[k].z);
  if (!sun.identity) {
    Frame f;
    f.u = sun.u;
    f.n = sun.n;
    f.v = sun.v;
    f.identity = false;
    d = qs::to_world(f, d);
  }
  out[i] = make_float4(d.x, d.y, d.z, 0.0f);
}

// Largest tan(angle from +y) of a pool, as float bits (non-negative floats
// order like their bit patterns); +inf when some direction has y <= 0.
__global__ void pool_tan_kernel(const float4* pool, int n, unsigned* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  float t = 0.0f;
  if (i < n) {
    const float4 q = pool[i];
    t = q.y > 0.0f ? sqrtf(q.x * q.x + q.z * q.z) / q.y : __int_as_float(0x7f800000);
  }
  for (int off = 16; off > 0; off >>= 1) t = fmaxf(t, __shfl_down_sync(0xffffffffu, t, off));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(t));
}

// Counts the xyz vectors whose squared length lies outside [0.25, 4] or is
// NaN (one warp-aggregated atomic per warp).
__global__ void count_non_unit_kernel(const float* xyz, int n, unsigned* bad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  bool b = false;
  if (i < n) {
    const float x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
    const float s = x * x + y * y + z * z;
    b = !(s >= 0.25f && s <= 4.0f);
  }
  const unsigned votes = __ballot_sync(0xffffffffu, b);
  if ((threadIdx.x & 31) == 0 && votes) atomicAdd(bad, (unsigned)__popc(votes));
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

cudaError_t launch_offsets_all(int* out, const long long* seg, int heliostats, long long total, uint32_t seed, int pool,
                               cudaStream_t stream) {
  if (total <= 0 || heliostats <= 0) return cudaSuccess;
  offsets_all_kernel<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(out, seg, heliostats, seed, pool);
  return cudaGetLastError();
}

cudaError_t launch_trace_pools(const float4* samples, const float4* perturbations, int n, int n_out,
                               const SunFrame& sun, float4* out, float4* pert_out, cudaStream_t stream) {
  if (n <= 0 || n_out <= 0) return cudaSuccess;
  trace_pools_kernel<<<(n_out + 255) / 256, 256, 0, stream>>>(samples, perturbations, n, n_out, sun, out, pert_out);
  return cudaGetLastError();
}

cudaError_t launch_pool_tan(const float4* pool, int n, unsigned* out, cudaStream_t stream) {
  if (n <= 0) return cudaSuccess;
  pool_tan_kernel<<<(n + 255) / 256, 256, 0, stream>>>(pool, n, out);
  return cudaGetLastError();
}

cudaError_t launch_count_non_unit(const float* xyz, int n, unsigned* bad, cudaStream_t stream) {
  if (n <= 0) return cudaSuccess;
  count_non_unit_kernel<<<(n + 255) / 256, 256, 0, stream>>>(xyz, n, bad);
  return cudaGetLastError();
}

cudaError_t launch_xyz_to_float4(const float* xyz, float4* out, int n, cudaStream_t stream) {
  if (n <= 0) return cudaSuccess;
  xyz_to_float4_kernel<<<(n + 255) / 256, 256, 0, stream>>>(xyz, out, n);
  return cudaGetLastError();
}

}  // namespace qm
