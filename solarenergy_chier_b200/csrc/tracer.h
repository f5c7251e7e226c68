// Launchers of the sm_100a kernels, one symbol per compiled variant.
#pragma once

#include <cuda_runtime.h>

#include "device_scene.h"

namespace qm {

// tracer.cu built with FMA contraction (production) and without it
// (every float operation rounded as the CPU oracle rounds it).
// out: 0 flux into the receiver images, 1 per-ray outcome codes
// (TraceParams::records), 2 bilinear deposit plus hit bits (TraceParams::hit_bits),
// 3 hit bits alone.  work_counter: one device word for flux launches of the
// persistent build (launch_trace_fast_ps), which zeroes it; the other builds
// ignore it.  It is a kernel argument of that build alone, not a TraceParams
// field: growing the kernels' parameter block changed the register
// allocation of every build and cost 2.5-3.7 % of their throughput.
cudaError_t launch_trace_fast(const TraceParams& p, int out, cudaStream_t stream,
                              unsigned long long* work_counter = nullptr);
cudaError_t launch_trace_exact(const TraceParams& p, int out, cudaStream_t stream,
                              unsigned long long* work_counter = nullptr);
// Production build limited to 64 registers (four 256-thread blocks per SM).
cudaError_t launch_trace_fast4(const TraceParams& p, int out, cudaStream_t stream,
                              unsigned long long* work_counter = nullptr);
// Production build in other launch shapes (the autotuner's candidates):
// 32-iteration and 128-iteration warp chunks, two-warp blocks.
cudaError_t launch_trace_fast_c32(const TraceParams& p, int out, cudaStream_t stream,
                              unsigned long long* work_counter = nullptr);
cudaError_t launch_trace_fast_c128(const TraceParams& p, int out, cudaStream_t stream,
                              unsigned long long* work_counter = nullptr);
cudaError_t launch_trace_fast_t64(const TraceParams& p, int out, cudaStream_t stream,
                              unsigned long long* work_counter = nullptr);
int trace_chunk_rays_fast_c32();
int trace_chunk_rays_fast_c128();
int trace_chunk_rays_fast_t64();
// Persistent launch shape: resident one-warp blocks taking warp chunks from a
// work counter in flux launches (without one it launches one warp per chunk).
cudaError_t launch_trace_fast_ps(const TraceParams& p, int out, cudaStream_t stream,
                              unsigned long long* work_counter = nullptr);
int trace_chunk_rays_fast_ps();
// Production build with the arithmetic after the receiver's decisions
// approximated (hit point, pixel position, energy).
cudaError_t launch_trace_rx(const TraceParams& p, int out, cudaStream_t stream,
                              unsigned long long* work_counter = nullptr);
int trace_chunk_rays_rx();
// Production build with approximate per-ray arithmetic after the shadow test
// (FMA contraction, hardware reciprocal square root, approximate divisions).
cudaError_t launch_trace_approx(const TraceParams& p, int out, cudaStream_t stream,
                              unsigned long long* work_counter = nullptr);
int trace_chunk_rays_approx();
cudaError_t launch_facets_approx(const DevTask& task, float3* origins, float3* normals, cudaStream_t stream);
// Rays per warp chunk; TraceParams::facet_prefix counts chunks per task.
int trace_chunk_rays_fast();
int trace_chunk_rays_exact();
int trace_chunk_rays_fast4();

// Micro-facet centres and normals of one heliostat, from the same device
// function the tracer evaluates per facet.
cudaError_t launch_facets_fast(const DevTask& task, float3* origins, float3* normals, cudaStream_t stream);
cudaError_t launch_facets_exact(const DevTask& task, float3* origins, float3* normals, cudaStream_t stream);
cudaError_t launch_facets_fast4(const DevTask& task, float3* origins, float3* normals, cudaStream_t stream);

}  // namespace qm
