// Compensated, fixed-order per-heliostat FP64 power of a trace launch
// (power.cu): adds the per-chunk partials the tracer wrote to
// TraceParams::chunk_power into TraceParams::power.
#pragma once

#include <cuda_runtime.h>

#include "device_scene.h"

namespace qm {
cudaError_t launch_power_reduce(const TraceParams& p, cudaStream_t stream);
}  // namespace qm
