// Internal state of a batch (qmcrt_batch), shared by batch.cpp and diff.cpp.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "prep.h"
#include "runtime.h"

struct qmcrt_batch {
  int device = 0;
  struct Instance {
    qmcrt_scene* scene;
    float3 sun;
    int grid_base, recv_base, power_base, task_base;
    long long pool_base;   // first float4 of its world-space pool (P + L entries)
  };
  std::vector<Instance> inst;
  std::vector<long long> image_offset;  // per instance-receiver, into d_images
  std::vector<int2> image_shape;        // (width, height)
  std::vector<qm::DevGrid> grids;
  std::vector<qm::DevReceiver> receivers;
  std::vector<qm::DevTask> tasks;
  std::vector<qm::PrepItem> items;
  qrt::DBuf d_grids, d_receivers, d_tasks, d_prefix, d_items, d_rot;
  qrt::DBuf d_bound, d_hsub, d_subv, d_verts, d_sub_free, d_sub_cand, d_sub_frames;  // per instance-grid slices
  qrt::DBuf d_images, d_power, d_diag, d_pools;
  qrt::DBuf d_chunk_power;  // per-chunk FP64 power partials of a launch (sized with the chunk prefix)
  qrt::DBuf d_work;         // work counter of persistent flux launches
  int light_begin = 0, light_end = 0, max_lights = 0;
  long long total_chunks = -1;  // for the current light range; -1 = prefix not built
  int mode = 0;                 // 0 production, 1 exact, 2 production at 64 registers, 3 approximate math
  int shape = 0;                // launch shape of the production build (qmcrt_batch_set_launch_shape)
  uint32_t* hit_bits = nullptr;  // output of bilinear-deposit launches (owned by the caller)
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;

  void drop_graph() {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph) cudaGraphDestroy(graph);
    graph_exec = nullptr;
    graph = nullptr;
  }
  ~qmcrt_batch() {
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    cudaDeviceSynchronize();
    drop_graph();
    for (qrt::DBuf* b : {&d_grids, &d_receivers, &d_tasks, &d_prefix, &d_items, &d_rot, &d_bound, &d_hsub, &d_subv,
                    &d_verts, &d_sub_free, &d_sub_cand, &d_sub_frames, &d_images, &d_power, &d_diag, &d_pools,
                    &d_chunk_power, &d_work})
      b->release();
    cudaSetDevice(prev);
  }
};

namespace qrt {

// Uploads the tasks and preparation items and prepares every instance for
// its sun on the device (normals, frames, parallelograms, records, pools).
void batch_prepare(qmcrt_batch* b, cudaStream_t st);
// Chunk prefix of the tasks for the current light range.
void batch_build_prefix(qmcrt_batch* b);
// One trace launch over the tasks' warp chunks [chunk_begin, chunk_end)
// (chunk_end < 0: to the last); out as qm::launch_trace_*.
cudaError_t batch_launch(qmcrt_batch* b, cudaStream_t st, int out, long long chunk_begin = 0, long long chunk_end = -1);

}  // namespace qrt
