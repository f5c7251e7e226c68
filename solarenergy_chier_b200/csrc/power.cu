// Per-heliostat FP64 power of a trace launch, summed with compensation and
// in a fixed order.
//
// The tracer's warps write one FP64 partial per warp chunk (the sum of its
// rays' energies: per-lane sums of at most 64 float energies, exact in
// double for the magnitudes of one heliostat, then a warp shuffle tree) to
// TraceParams::chunk_power.  This kernel adds each task's partials, one warp
// per task: every lane runs a Neumaier-compensated sum over a lane-strided
// subset, the 32 (sum, compensation) pairs merge by error-free two-sums down
// a fixed shuffle tree, and lane 0 adds the rounded result to the task's
// power slot.  The order never depends on scheduling, so a launch's
// per-heliostat powers are the same on every run, and the total error stays
// at the last bit of the double result instead of growing with the number
// of chunks, as one double atomic per chunk let it.
#include "device_scene.h"
#include "power.h"

namespace qm {
namespace {

__device__ __forceinline__ void neumaier(double& s, double& c, double x) {
  const double t = s + x;
  c += fabs(s) >= fabs(x) ? (s - t) + x : (x - t) + s;
  s = t;
}

__global__ void power_reduce_kernel(TraceParams p) {
  const long long t = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (t >= p.num_tasks) return;
  const long long c0 = max(__ldg(p.facet_prefix + t), p.chunk_begin);
  const long long c1 = min(__ldg(p.facet_prefix + t + 1), p.total_facets);
  if (c1 <= c0) return;  // warp-uniform
  double s = 0.0, c = 0.0;
  for (long long k = c0 + lane; k < c1; k += 32) neumaier(s, c, p.chunk_power[k - p.chunk_begin]);
  for (int off = 16; off > 0; off >>= 1) {
    const double s2 = __shfl_down_sync(0xffffffffu, s, off);
    const double c2 = __shfl_down_sync(0xffffffffu, c, off);
    const double sum = s + s2;
    const double bb = sum - s;
    const double err = (s - (sum - bb)) + (s2 - bb);  // two-sum: s + s2 = sum + err exactly
    s = sum;
    c += c2 + err;
  }
  if (lane == 0) {
    const double v = s + c;
    if (v != 0.0) atomicAdd(p.power + p.tasks[t].power_slot, v);
  }
}

}  // namespace

cudaError_t launch_power_reduce(const TraceParams& p, cudaStream_t stream) {
  if (!p.chunk_power || p.num_tasks <= 0) return cudaSuccess;
  const int threads = 128;
  const long long blocks = ((long long)p.num_tasks * 32 + threads - 1) / threads;
  power_reduce_kernel<<<(unsigned)blocks, threads, 0, stream>>>(p);
  return cudaGetLastError();
}

}  // namespace qm
