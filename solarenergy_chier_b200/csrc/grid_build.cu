// GPU construction of a grid's cell lists: the reference's
// RectangleGrid::CGridHelioMatch (Scene/DataStructure/Grid/RectangleGrid.cu:62-117),
// which the host restates in match_grid (csrc/scene.cpp), as a count / scan /
// fill / sort pass over the heliostats.
//
// Every heliostat covers the cells of its box pos +- |size| / 2 (|size|:
// the length of the size vector, so the box holds the heliostat in any
// orientation), computed with the same explicitly rounded float operations
// as the host, and is listed in each of them.  Cell lists come out in
// heliostat order, as the host's (the fill scatters with atomics, then one
// thread per cell sorts its short list), so the device lists equal the host
// lists entry for entry.
#include "grid_build.h"

#include "vecmath.h"

namespace qm {
namespace {

__device__ __forceinline__ bool helio_cells(const GridBuildParams& p, int i, int3& lo_c, int3& hi_c) {
  const float4 ps = p.pos_radius[i];
  const float3 pos = make_float3(ps.x, ps.y, ps.z);
  const float r = ps.w;
  const float3 lo = qs::subs(pos, r), hi = qs::adds(pos, r);
  lo_c = qs::trunc3(qs::cdiv(qs::sub(lo, p.pos), p.interval));
  hi_c = qs::trunc3(qs::cdiv(qs::sub(hi, p.pos), p.interval));
  lo_c = make_int3(max(0, lo_c.x), max(0, lo_c.y), max(0, lo_c.z));
  hi_c = make_int3(min(p.cells.x - 1, hi_c.x), min(p.cells.y - 1, hi_c.y), min(p.cells.z - 1, hi_c.z));
  return lo_c.x <= hi_c.x && lo_c.y <= hi_c.y && lo_c.z <= hi_c.z;
}

__global__ void count_kernel(GridBuildParams p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.num_heliostats) return;
  int3 a, b;
  if (!helio_cells(p, i, a, b)) return;
  for (int x = a.x; x <= b.x; ++x)
    for (int y = a.y; y <= b.y; ++y)
      for (int z = a.z; z <= b.z; ++z) atomicAdd(p.counts + ((long long)x * p.cells.y + y) * p.cells.z + z, 1);
}

// Exclusive scan of the counts into the cell ranges, one block walking the
// cells 1,024 at a time with a running carry.
__global__ void scan_kernel(GridBuildParams p, long long ncell) {
  __shared__ int buf[1024];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (long long base = 0; base < ncell; base += 1024) {
    const long long c = base + threadIdx.x;
    const int v = c < ncell ? p.counts[c] : 0;
    buf[threadIdx.x] = v;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
      const int t = threadIdx.x >= off ? buf[threadIdx.x - off] : 0;
      __syncthreads();
      buf[threadIdx.x] += t;
      __syncthreads();
    }
    if (c < ncell) {
      const int end = carry + buf[threadIdx.x];
      p.ranges[c] = make_int2(end - v, end);
      p.counts[c] = 0;  // reused as the fill cursor
    }
    __syncthreads();
    if (threadIdx.x == 1023) carry += buf[1023];
    __syncthreads();
  }
  if (threadIdx.x == 0) *p.total = carry;
}

__global__ void fill_kernel(GridBuildParams p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.num_heliostats) return;
  int3 a, b;
  if (!helio_cells(p, i, a, b)) return;
  const int2 sub = p.subs[i];  // first sub-heliostat, count
  for (int x = a.x; x <= b.x; ++x)
    for (int y = a.y; y <= b.y; ++y)
      for (int z = a.z; z <= b.z; ++z) {
        const long long cell = ((long long)x * p.cells.y + y) * p.cells.z + z;
        const int k = p.ranges[cell].x + atomicAdd(p.counts + cell, 1);
        p.entries[k] = make_int4(i, sub.x, sub.y, 0);
      }
}

__global__ void sort_kernel(GridBuildParams p, long long ncell) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  const int2 r = p.ranges[c];
  for (int k = r.x + 1; k < r.y; ++k) {
    const int4 e = p.entries[k];
    int j = k - 1;
    while (j >= r.x && p.entries[j].x > e.x) {
      p.entries[j + 1] = p.entries[j];
      --j;
    }
    p.entries[j + 1] = e;
  }
}

}  // namespace

cudaError_t launch_grid_count(const GridBuildParams& p, cudaStream_t stream) {
  const long long ncell = (long long)p.cells.x * p.cells.y * p.cells.z;
  if (ncell <= 0) return cudaErrorInvalidValue;
  cudaError_t e = cudaMemsetAsync(p.counts, 0, (size_t)ncell * sizeof(int), stream);
  if (e != cudaSuccess) return e;
  if (p.num_heliostats > 0) count_kernel<<<(p.num_heliostats + 127) / 128, 128, 0, stream>>>(p);
  scan_kernel<<<1, 1024, 0, stream>>>(p, ncell);
  return cudaGetLastError();
}

cudaError_t launch_grid_fill(const GridBuildParams& p, cudaStream_t stream) {
  const long long ncell = (long long)p.cells.x * p.cells.y * p.cells.z;
  if (ncell <= 0) return cudaErrorInvalidValue;
  if (p.num_heliostats > 0) fill_kernel<<<(p.num_heliostats + 127) / 128, 128, 0, stream>>>(p);
  sort_kernel<<<(unsigned)((ncell + 255) / 256), 256, 0, stream>>>(p, ncell);
  return cudaGetLastError();
}

}  // namespace qm
