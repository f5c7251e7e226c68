// Differentiable forward / adjoint kernels (diff.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "device_scene.h"
#include "prep.h"

namespace qm {

constexpr int kDiffParams = 4;  // per heliostat: aim offset u, v (m); normal offset u, v (rad)

// A float and its derivatives with respect to one heliostat's parameters.
struct Dual {
  float v;
  float d[kDiffParams];
};
struct Dual3 {
  Dual x, y, z;
};

// Per task: the heliostat normal and its facet frame as functions of the
// heliostat's parameters (value + tangents), for the adjoint.
struct DiffTask {
  Dual3 n, u, fn, v;  // normal; frame (u, n, v) of the facet transform
  int identity;
};

struct BackwardParams {
  const DevTask* tasks;
  const DiffTask* dtasks;
  const DevReceiver* receivers;   // images hold P = G * dL/dF (the smoothed residual)
  const long long* chunk_prefix;  // as TraceParams::facet_prefix
  int num_tasks;
  long long total_chunks;         // end of the launch's chunks (chunks [chunk_begin, total_chunks))
  long long chunk_begin;
  int light_begin, light_end;
  int lights_q32, lights_r32;
  // one word per warp iteration of the launch (chunk - chunk_begin): the
  // forward's bilinear-deposit launch, or a hit-bit launch over the same chunks
  const uint32_t* hit_bits;
  double* grad;                   // kDiffParams per power slot
};

cudaError_t launch_diff_prep(const PrepItem* items, int n, const DevTask* tasks, DiffTask* out, cudaStream_t stream);
cudaError_t launch_diff_backward(const BackwardParams& p, cudaStream_t stream);

// Separable normalised Gaussian of `radius` taps each side (weights[0..radius])
// along rows (columns wrap when `wrap_cols`) then columns (zero outside).
cudaError_t launch_gauss(const float* in, float* tmp, float* out, int width, int height, const float* weights,
                         int radius, bool wrap_cols, cudaStream_t stream);
// out[i] = (float)in[i].
cudaError_t launch_round_deposit(const double* in, float* out, long long n, cudaStream_t stream);
// resid = 2 (flux - target); *loss += sum (flux - target)^2 (FP64).
cudaError_t launch_loss(const float* flux, const float* target, float* resid, long long n, double* loss,
                        cudaStream_t stream);

}  // namespace qm
