// GPU construction of a grid's cell lists (grid_build.cu).
#pragma once

#include <cuda_runtime.h>

namespace qm {

struct GridBuildParams {
  float3 pos, interval;  // grid origin and cell size
  int3 cells;
  int num_heliostats;
  const float4* pos_radius;  // per heliostat of the grid: position, |size| / 2
  const int2* subs;          // per heliostat: first sub-heliostat (grid-local), count
  int* counts;               // scratch: one int per cell
  int2* ranges;              // out: [begin, end) of each cell's entries
  int4* entries;             // out: (heliostat, first sub-heliostat, count, 0), heliostat order per cell
  int* total;                // out: number of entries
};

// Counts and ranges (ranges, total); then, once `entries` holds *total
// entries, the entries themselves.
cudaError_t launch_grid_count(const GridBuildParams& p, cudaStream_t stream);
cudaError_t launch_grid_fill(const GridBuildParams& p, cudaStream_t stream);

}  // namespace qm
