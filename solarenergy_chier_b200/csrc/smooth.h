#pragma once

#include <cuda_runtime.h>

namespace qm {

// Floats per heap per thread: int((2r+1)^2 * ratio) + 1, the reference's
// heap_size (Tool/Smoother/ImageSmoother.cu:103).
int smooth_heap_stride(int radius, float ratio);

// Trimmed mean of `src` into `dst` (distinct buffers), 16x16 blocks.
cudaError_t launch_trimmed_mean(const float* src, float* dst, int width, int height, int radius, float ratio,
                                cudaStream_t stream);

}  // namespace qm
