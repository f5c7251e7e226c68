// Batched tracing (include/qmcrt.h, qmcrt_batch_*): many (scene, sun)
// instances traced by one kernel launch.
//
// Every instance owns its sun-dependent data -- heliostat normals and facet
// frames (in its tasks), sub-heliostat parallelograms and traversal records
// (per grid), the world-space sun-shape pool, receiver images and FP64
// per-heliostat powers -- and shares the rest with its scene: grid cell
// lists, focus-flat local frames, facet pool offsets, the slope-error pool.
// The sun-dependent data is prepared on the device (csrc/prep.cu) for all
// instances at once; the host only lays out buffers and task templates.
// A trace is one launch over the tasks of all instances (tasks are ordered
// instance by instance, so the grid and image data a warp touches stays
// within one instance), optionally replayed from a captured CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "batch_state.h"
#include "tracer.h"
#include "vecmath.h"

using namespace qrt;

namespace {

qmcrt_batch* batch_checked(qmcrt_batch* b) {
  if (!b) invalid("batch is NULL");
  return b;
}

float3 sun_of(const float* dirs, int k) {
  const float3 d = make_float3(dirs[3 * k], dirs[3 * k + 1], dirs[3 * k + 2]);
  if (!std::isfinite(d.x) || !std::isfinite(d.y) || !std::isfinite(d.z) || (d.x == 0 && d.y == 0 && d.z == 0))
    invalid("sun direction " + std::to_string(k) + " must be finite and non-zero");
  return d;
}

qm::SunFrame sun_frame(float3 sun) {
  // Frame of -sun_dir, as the plain path builds it.
  const qm::Frame f = qm::make_frame(qm::neg(sun), false);
  qm::SunFrame s;
  s.u = f.u;
  s.n = f.n;
  s.v = f.v;
  s.identity = f.identity ? 1 : 0;
  return s;
}

}  // namespace

namespace qrt {

void batch_prepare(qmcrt_batch* b, cudaStream_t st) {
  for (size_t k = 0; k < b->inst.size(); ++k) {
    const auto& I = b->inst[k];
    const int H = (int)I.scene->model.heliostats.size();
    float3 axis;
    float tan_world;
    sun_cone(I.sun, I.scene->sun_shape_tan, axis, tan_world);
    const float block_theta = tan_world < 0.0f || I.scene->slope_angle < 0.0f
                                  ? -1.0f
                                  : std::atan(tan_world) + 2.0f * I.scene->slope_angle;
    for (int h = 0; h < H; ++h) {
      qm::PrepItem& it = b->items[I.task_base + h];
      it.sun_dir = I.sun;
      it.shadow_axis = axis;
      it.shadow_tan = tan_world;
      it.block_theta = block_theta;
    }
  }
  cuda_check(cudaMemcpyAsync(b->d_tasks.p, b->tasks.data(), b->tasks.size() * sizeof(qm::DevTask),
                             cudaMemcpyHostToDevice, st),
             "task upload");
  cuda_check(cudaMemcpyAsync(b->d_items.p, b->items.data(), b->items.size() * sizeof(qm::PrepItem),
                             cudaMemcpyHostToDevice, st),
             "prep upload");
  cuda_check(qm::launch_prep(b->d_items.as<qm::PrepItem>(), (int)b->items.size(), b->d_tasks.as<qm::DevTask>(), st),
             "prep kernel");
  int max_sub = 0;
  for (const auto& it : b->items) max_sub = std::max(max_sub, it.num_sub);
  cuda_check(qm::launch_shadow_flags(b->d_items.as<qm::PrepItem>(), (int)b->items.size(), max_sub,
                                     b->d_tasks.as<qm::DevTask>(), b->d_grids.as<qm::DevGrid>(), st),
             "shadow flags");
  std::vector<qm::PoolRotation> rot(b->inst.size());
  int max_out = 0;
  for (size_t k = 0; k < b->inst.size(); ++k) {
    const auto& I = b->inst[k];
    const int L = I.scene->model.config.num_per_sunshape_group;
    rot[k].in = I.scene->d_samples.as<float4>();
    rot[k].out = b->d_pools.as<float4>() + I.pool_base;
    rot[k].n = I.scene->pool_size;
    rot[k].n_out = I.scene->pool_size + L;
    rot[k].sun = sun_frame(I.sun);
    max_out = std::max(max_out, rot[k].n_out);
  }
  upload(b->d_rot, rot);
  for (size_t k0 = 0; k0 < rot.size(); k0 += 65535) {
    const int n = (int)std::min<size_t>(65535, rot.size() - k0);
    cuda_check(qm::launch_rotate_pools(b->d_rot.as<qm::PoolRotation>() + k0, n, max_out, st), "pool rotation");
  }
  cuda_check(cudaStreamSynchronize(st), "batch preparation");
}

void batch_build_prefix(qmcrt_batch* b) {
  const long long nl = b->light_end - b->light_begin;
  const long long chunk = chunk_rays_for(b->mode, b->shape, 0);
  std::vector<long long> prefix(b->tasks.size() + 1, 0);
  for (size_t i = 0; i < b->tasks.size(); ++i) {
    const long long rays = (long long)b->tasks[i].num_facets * nl;
    if (rays > kMaxTaskRays) invalid("a heliostat's micro-facets x lights must stay below 2^31 - 2^16 rays per launch");
    prefix[i + 1] = prefix[i] + (rays + chunk - 1) / chunk;
  }
  upload(b->d_prefix, prefix);
  b->total_chunks = prefix.back();
  // allocated here, before any graph capture of the launch
  chunk_power_buffer(b->d_chunk_power, b->total_chunks);
  if (b->d_work.bytes < sizeof(unsigned long long)) b->d_work.alloc(sizeof(unsigned long long));
}

cudaError_t batch_launch(qmcrt_batch* b, cudaStream_t st, int out, long long chunk_begin, long long chunk_end) {
  qm::TraceParams p{};
  p.grids = b->d_grids.as<qm::DevGrid>();
  p.receivers = b->d_receivers.as<qm::DevReceiver>();
  p.tasks = b->d_tasks.as<qm::DevTask>();
  p.facet_prefix = b->d_prefix.as<long long>();
  p.num_tasks = (int)b->tasks.size();
  p.chunk_begin = chunk_begin;
  p.total_facets = chunk_end < 0 ? b->total_chunks : std::min(chunk_end, b->total_chunks);
  p.light_begin = b->light_begin;
  p.light_end = b->light_end;
  p.power = b->d_power.as<double>();
  p.diag = b->d_diag.as<unsigned long long>();
  p.hit_bits = b->hit_bits;
  if (out == 0 || out == 2) p.chunk_power = b->d_chunk_power.as<double>();
  // the prefix is laid out for the flux kernel's chunk size
  if (chunk_rays_for(b->mode, b->shape, out) != chunk_rays_for(b->mode, b->shape, 0)) return cudaErrorInvalidValue;
  return launch_trace_mode(b->mode, p, out, st, b->shape, out == 0 ? b->d_work.as<unsigned long long>() : nullptr);
}

}  // namespace qrt

namespace {

void clear_async(qmcrt_batch* b, cudaStream_t st) {
  cuda_check(cudaMemsetAsync(b->d_images.p, 0, b->d_images.bytes, st), "clear");
  cuda_check(cudaMemsetAsync(b->d_power.p, 0, b->d_power.bytes, st), "clear");
}

const qmcrt_batch::Instance& instance(const qmcrt_batch* b, int k) {
  if (k < 0 || k >= (int)b->inst.size()) invalid("instance index out of range");
  return b->inst[k];
}

}  // namespace

extern "C" {

int qmcrt_batch_create(qmcrt_scene* const* scenes, int n_scenes, const int* scene_of, const float* sun_dirs, int n,
                       qmcrt_batch** out) {
  return guarded([&] {
    if (!out) invalid("output handle is NULL");
    *out = nullptr;
    if (!scenes || n_scenes <= 0 || !scene_of || !sun_dirs || n <= 0) invalid("empty or NULL batch description");
    for (int i = 0; i < n_scenes; ++i) checked(scenes[i]);
    for (int i = 1; i < n_scenes; ++i)
      if (scenes[i]->device != scenes[0]->device) invalid("all scenes of a batch must live on one device");
    auto b = std::make_unique<qmcrt_batch>();
    b->device = scenes[0]->device;
    DeviceGuard guard(b->device);

    // Layout: element offsets of every instance's slices in the batch buffers.
    struct GridSlot {
      long long bound, hsub, sub;  // first float4, first int4, first sub-heliostat
    };
    std::vector<GridSlot> grid_slot;
    struct ItemSlot {
      int grid;             // batch grid index
      long long local;      // grid-local heliostat index
    };
    std::vector<ItemSlot> item_slot;
    long long n_hsub = 0, n_sub = 0, n_img = 0, n_pool = 0;
    int n_power = 0;
    b->max_lights = 1 << 30;
    for (int k = 0; k < n; ++k) {
      if (scene_of[k] < 0 || scene_of[k] >= n_scenes) invalid("instance scene index out of range");
      qmcrt_scene* s = scenes[scene_of[k]];
      const qm::SceneModel& m = s->model;
      qmcrt_batch::Instance I{};
      I.scene = s;
      I.sun = sun_of(sun_dirs, k);
      I.grid_base = (int)b->grids.size();
      I.recv_base = (int)b->receivers.size();
      I.power_base = n_power;
      I.task_base = (int)b->tasks.size();
      I.pool_base = n_pool;
      const int L = m.config.num_per_sunshape_group;
      b->max_lights = std::min(b->max_lights, L);
      n_pool += s->pool_size + L;
      for (size_t g = 0; g < m.grids.size(); ++g) {
        grid_slot.push_back({5 * n_hsub, n_hsub, n_sub});
        n_hsub += m.grids[g].num_heliostats;
        n_sub += m.grids[g].num_subheliostats;
        b->grids.push_back(s->grids[g]);  // cell lists shared; sun-dependent pointers set below
      }
      for (size_t r = 0; r < m.receivers.size(); ++r) {
        const qm::DevReceiver& dr = s->receivers[r];
        b->image_offset.push_back(n_img);
        b->image_shape.push_back(dr.resolution);
        n_img += std::max<long long>((long long)dr.resolution.x * dr.resolution.y, 1);
        b->receivers.push_back(dr);  // image pointer set below
      }
      const int H = (int)m.heliostats.size();
      for (int h = 0; h < H; ++h) {
        const qm::HeliostatModel& hm = m.heliostats[h];
        const qm::GridModel& gm = m.grids[hm.grid];
        qm::DevTask t = s->templates[h];
        t.grid = I.grid_base + hm.grid;
        t.receiver = I.recv_base + gm.receiver;
        t.power_slot = I.power_base + h;
        b->tasks.push_back(t);  // samples pointer set below; normal and frames by the prep kernel
        qm::PrepItem it{};
        it.task = I.task_base + h;
        it.num_sub = hm.num_sub;
        it.sub_first = hm.sub_begin;
        it.focus = hm.focus;
        b->items.push_back(it);
        item_slot.push_back({t.grid, h - gm.start_heliostat});
      }
      n_power += H;
      b->inst.push_back(I);
    }
    b->d_bound.alloc(std::max<long long>(5 * n_hsub, 1) * sizeof(float4));
    b->d_hsub.alloc(std::max<long long>(n_hsub, 1) * sizeof(int4));
    b->d_subv.alloc(std::max<long long>(3 * n_sub, 1) * sizeof(float4));
    b->d_verts.alloc(std::max<long long>(3 * n_sub, 1) * sizeof(float3));
    b->d_sub_free.alloc(std::max<long long>(n_sub, 1) * sizeof(int));
    b->d_sub_cand.alloc(std::max<long long>(n_sub, 1) * qm::kMaxCandidates * sizeof(int));
    b->d_sub_frames.alloc(std::max<long long>(n_sub, 1) * 6 * sizeof(float4));
    b->d_images.alloc(std::max<long long>(n_img, 1) * sizeof(float));
    b->d_power.alloc(std::max(n_power, 1) * sizeof(double));
    b->d_pools.alloc(std::max<long long>(n_pool, 1) * sizeof(float4));
    b->d_diag.alloc(qm::kDiagSlots * sizeof(unsigned long long));
    cuda_check(cudaMemset(b->d_images.p, 0, b->d_images.bytes), "cudaMemset");
    cuda_check(cudaMemset(b->d_power.p, 0, b->d_power.bytes), "cudaMemset");
    cuda_check(cudaMemset(b->d_diag.p, 0, b->d_diag.bytes), "cudaMemset");
    for (size_t g = 0; g < b->grids.size(); ++g) {
      b->grids[g].bound = b->d_bound.as<float4>() + grid_slot[g].bound;
      b->grids[g].hsub = b->d_hsub.as<int4>() + grid_slot[g].hsub;
      b->grids[g].subv = b->d_subv.as<float4>() + 3 * grid_slot[g].sub;
      b->grids[g].sub_free = b->d_sub_free.as<int>() + grid_slot[g].sub;
      b->grids[g].sub_cand = b->d_sub_cand.as<int>() + grid_slot[g].sub * qm::kMaxCandidates;
      b->grids[g].sub_frames = b->d_sub_frames.as<float4>() + grid_slot[g].sub * 6;
    }
    for (size_t r = 0; r < b->receivers.size(); ++r) b->receivers[r].image = b->d_images.as<float>() + b->image_offset[r];
    for (const auto& I : b->inst)
      for (int h = 0; h < (int)I.scene->model.heliostats.size(); ++h)
        b->tasks[I.task_base + h].samples = b->d_pools.as<float4>() + I.pool_base;
    for (size_t i = 0; i < b->items.size(); ++i) {
      qm::PrepItem& it = b->items[i];
      const GridSlot& gs = grid_slot[item_slot[i].grid];
      const long long sub = gs.sub + it.sub_first;
      it.verts = b->d_verts.as<float3>() + 3 * sub;
      it.subv = b->d_subv.as<float4>() + 3 * sub;
      it.sub_free = b->d_sub_free.as<int>() + sub;
      it.sub_cand = b->d_sub_cand.as<int>() + sub * qm::kMaxCandidates;
      it.sub_frames = b->d_sub_frames.as<float4>() + sub * 6;
      it.bound = b->d_bound.as<float4>() + gs.bound + 5 * item_slot[i].local;
      it.hsub = b->d_hsub.as<int4>() + gs.hsub + item_slot[i].local;
    }
    upload(b->d_grids, b->grids);
    upload(b->d_receivers, b->receivers);
    b->d_tasks.alloc(b->tasks.size() * sizeof(qm::DevTask));
    b->d_items.alloc(b->items.size() * sizeof(qm::PrepItem));
    b->light_begin = 0;
    b->light_end = b->max_lights;
    batch_prepare(b.get(), 0);
    *out = b.release();
  });
}

void qmcrt_batch_free(qmcrt_batch* b) { delete b; }

int qmcrt_batch_set_suns(qmcrt_batch* b, const float* sun_dirs, void* stream) {
  return guarded([&] {
    batch_checked(b);
    if (!sun_dirs) invalid("sun directions are NULL");
    for (size_t k = 0; k < b->inst.size(); ++k) b->inst[k].sun = sun_of(sun_dirs, (int)k);
    DeviceGuard guard(b->device);
    batch_prepare(b, static_cast<cudaStream_t>(stream));
  });
}

int qmcrt_batch_set_light_range(qmcrt_batch* b, int begin, int end) {
  return guarded([&] {
    batch_checked(b);
    if (begin < 0 || end < begin || end > b->max_lights) invalid("light range out of bounds");
    b->light_begin = begin;
    b->light_end = end;
    b->total_chunks = -1;
    b->drop_graph();
  });
}

int qmcrt_batch_set_math_mode(qmcrt_batch* b, int mode) {
  return guarded([&] {
    batch_checked(b);
    if (mode < 0 || mode > 4) invalid("math mode must be 0, 1, 2, 3 or 4");
    b->mode = mode;
    b->drop_graph();
  });
}

int qmcrt_batch_info(const qmcrt_batch* b, int* instances, int* tasks, long long* rays_per_trace) {
  return guarded([&] {
    if (!b) invalid("batch is NULL");
    if (instances) *instances = (int)b->inst.size();
    if (tasks) *tasks = (int)b->tasks.size();
    if (rays_per_trace) {
      long long r = 0;
      for (const auto& t : b->tasks) r += (long long)t.num_facets * (b->light_end - b->light_begin);
      *rays_per_trace = r;
    }
  });
}

int qmcrt_batch_trace(qmcrt_batch* b, void* stream) {
  return guarded([&] {
    batch_checked(b);
    if (b->light_end == b->light_begin) return;
    DeviceGuard guard(b->device);
    if (b->total_chunks < 0) batch_build_prefix(b);
    cuda_check(batch_launch(b, static_cast<cudaStream_t>(stream), 0), "batch trace");
  });
}

int qmcrt_batch_capture_graph(qmcrt_batch* b, int clear_first) {
  return guarded([&] {
    batch_checked(b);
    DeviceGuard guard(b->device);
    if (b->total_chunks < 0) batch_build_prefix(b);
    b->drop_graph();
    cudaStream_t st;
    cuda_check(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate");
    cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      if (clear_first) {
        cudaMemsetAsync(b->d_images.p, 0, b->d_images.bytes, st);
        cudaMemsetAsync(b->d_power.p, 0, b->d_power.bytes, st);
      }
      if (b->light_end > b->light_begin) batch_launch(b, st, 0);
      cudaError_t e2 = cudaStreamEndCapture(st, &b->graph);
      e = e2;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&b->graph_exec, b->graph, 0);
    cudaStreamDestroy(st);
    if (e != cudaSuccess) b->drop_graph();
    cuda_check(e, "graph capture");
  });
}

int qmcrt_batch_graph_launch(qmcrt_batch* b, void* stream) {
  return guarded([&] {
    batch_checked(b);
    if (!b->graph_exec) throw ApiError(QMCRT_ERR_STATE, "no captured graph (call qmcrt_batch_capture_graph)");
    DeviceGuard guard(b->device);
    cuda_check(cudaGraphLaunch(b->graph_exec, static_cast<cudaStream_t>(stream)), "graph launch");
  });
}

int qmcrt_batch_clear(qmcrt_batch* b, void* stream) {
  return guarded([&] {
    batch_checked(b);
    DeviceGuard guard(b->device);
    clear_async(b, static_cast<cudaStream_t>(stream));
  });
}

int qmcrt_batch_image(qmcrt_batch* b, int k, int receiver, float* out, int* width, int* height) {
  return guarded([&] {
    batch_checked(b);
    const auto& I = instance(b, k);
    const int nr = (int)I.scene->model.receivers.size();
    if (receiver < 0 || receiver >= nr) invalid("receiver index out of range");
    const int slot = I.recv_base + receiver;
    const int2 shape = b->image_shape[slot];
    if (width) *width = shape.x;
    if (height) *height = shape.y;
    if (!out) return;
    DeviceGuard guard(b->device);
    cuda_check(cudaMemcpy(out, b->d_images.as<float>() + b->image_offset[slot],
                          (size_t)shape.x * shape.y * sizeof(float), cudaMemcpyDeviceToHost),
               "image readback");
  });
}

int qmcrt_batch_power_fp64(qmcrt_batch* b, int k, double* per_heliostat, double* total) {
  return guarded([&] {
    batch_checked(b);
    const auto& I = instance(b, k);
    const int H = (int)I.scene->model.heliostats.size();
    std::vector<double> v(H);
    DeviceGuard guard(b->device);
    cuda_check(cudaMemcpy(v.data(), b->d_power.as<double>() + I.power_base, H * sizeof(double),
                          cudaMemcpyDeviceToHost),
               "power readback");
    if (per_heliostat) std::copy(v.begin(), v.end(), per_heliostat);
    if (total) {
      // Neumaier-compensated sum of the per-heliostat FP64 powers.
      double s = 0.0, c = 0.0;
      for (double x : v) {
        const double t = s + x;
        c += std::fabs(s) >= std::fabs(x) ? (s - t) + x : (x - t) + s;
        s = t;
      }
      *total = s + c;
    }
  });
}

int qmcrt_batch_debug_geometry(qmcrt_batch* b, int k, int grid, float* vertices, float* normals) {
  return guarded([&] {
    batch_checked(b);
    const auto& I = instance(b, k);
    const qm::SceneModel& m = I.scene->model;
    if (grid < 0 || grid >= (int)m.grids.size()) invalid("grid index out of range");
    DeviceGuard guard(b->device);
    cuda_check(cudaDeviceSynchronize(), "debug geometry");
    if (vertices) {
      // The prep kernel's float3 (B, A, C) table of this instance-grid starts
      // where the grid's parallelograms start.
      const qm::DevGrid& g = b->grids[I.grid_base + grid];
      const long long first = (g.subv - b->d_subv.as<float4>()) / 3;
      const size_t n = 3 * (size_t)m.grids[grid].num_subheliostats;
      cuda_check(cudaMemcpy(vertices, b->d_verts.as<float3>() + 3 * first, n * sizeof(float3),
                            cudaMemcpyDeviceToHost),
                 "vertex readback");
    }
    if (normals) {
      const int H = (int)m.heliostats.size();
      std::vector<qm::DevTask> t(H);
      cuda_check(cudaMemcpy(t.data(), b->d_tasks.as<qm::DevTask>() + I.task_base, H * sizeof(qm::DevTask),
                            cudaMemcpyDeviceToHost),
                 "task readback");
      for (int h = 0; h < H; ++h) {
        normals[3 * h] = t[h].normal.x;
        normals[3 * h + 1] = t[h].normal.y;
        normals[3 * h + 2] = t[h].normal.z;
      }
    }
  });
}

int qmcrt_batch_autotune_shapes(qmcrt_batch* b, void* stream, int* chosen, float* ms_per_shape) {
  return guarded([&] {
    batch_checked(b);
    DeviceGuard guard(b->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // The candidates are the production build's launch shapes: identical
    // per-ray arithmetic, different block widths, register budgets and warp
    // chunks.  Each is timed on the batch itself (its prefix rebuilt for the
    // shape's chunk size) and the fastest kept.  Images and powers are
    // cleared afterwards.
    int n_shapes = 0;
    qmcrt_launch_shapes(nullptr, nullptr, nullptr, &n_shapes);
    cudaEvent_t e0, e1;
    cuda_check(cudaEventCreate(&e0), "cudaEventCreate");
    cuda_check(cudaEventCreate(&e1), "cudaEventCreate");
    float best = 1e30f;
    int pick = 0;
    b->mode = 0;
    for (int k = 0; k < n_shapes; ++k) {
      b->shape = k;
      batch_build_prefix(b);
      cuda_check(batch_launch(b, st, 0), "autotune");  // warm-up
      cudaEventRecord(e0, st);
      cuda_check(batch_launch(b, st, 0), "autotune");
      cudaEventRecord(e1, st);
      cuda_check(cudaEventSynchronize(e1), "autotune");
      float t = 0.f;
      cudaEventElapsedTime(&t, e0, e1);
      if (ms_per_shape) ms_per_shape[k] = t;
      if (t < best) {
        best = t;
        pick = k;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->shape = pick;
    batch_build_prefix(b);
    b->drop_graph();
    clear_async(b, st);
    cuda_check(cudaStreamSynchronize(st), "autotune");
    if (chosen) *chosen = pick;
  });
}

int qmcrt_batch_autotune(qmcrt_batch* b, void* stream, int* chosen, float* ms) {
  float table[16] = {0};
  int pick = 0;
  const int rc = qmcrt_batch_autotune_shapes(b, stream, &pick, table);
  if (rc == QMCRT_OK) {
    if (chosen) *chosen = pick;
    if (ms) *ms = table[pick];
  }
  return rc;
}

int qmcrt_batch_set_launch_shape(qmcrt_batch* b, int shape) {
  return guarded([&] {
    batch_checked(b);
    int n_shapes = 0;
    qmcrt_launch_shapes(nullptr, nullptr, nullptr, &n_shapes);
    if (shape < 0 || shape >= n_shapes) invalid("launch shape out of range");
    b->shape = shape;
    b->total_chunks = -1;
    b->drop_graph();
  });
}

}  // extern "C"
