// Internal runtime shared by the C ABI units (capi.cpp, batch.cpp): error
// handling, device buffers and the scene state behind qmcrt_scene.  Not part
// of the public interface (include/qmcrt.h).
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "device_scene.h"
#include "qmcrt.h"
#include "scene.h"

namespace qm {
void set_last_error(const std::string& msg);
}  // namespace qm

namespace qrt {

struct ApiError : std::runtime_error {
  int code;
  ApiError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void cuda_check(cudaError_t e, const char* what) {
  if (e == cudaErrorMemoryAllocation) throw ApiError(QMCRT_ERR_NOMEM, std::string(what) + ": " + cudaGetErrorString(e));
  if (e != cudaSuccess) throw ApiError(QMCRT_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// Allocation gate: every allocation the C ABI makes for a scene, batch or
// differentiable pair (device buffers, pinned staging, the scene state
// itself) passes here first.  When failure injection is armed
// (QMCRT_INJECT_ALLOC_FAILURE=n in the environment when the library loads,
// or qmcrt_debug_fail_allocations(n)), the allocation after n successful
// ones fails with QMCRT_ERR_NOMEM as a real out-of-memory would, and
// injection disarms itself.  Defined in capi.cpp.
void alloc_gate(const char* what);

// Runs one C ABI call: exceptions become status codes, their message the
// thread's last error.
template <class F>
int guarded(F&& f) {
  try {
    f();
    qm::set_last_error("");
    return QMCRT_OK;
  } catch (const ApiError& e) {
    qm::set_last_error(e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    qm::set_last_error("host allocation failed");
    return QMCRT_ERR_NOMEM;
  } catch (const std::exception& e) {
    qm::set_last_error(e.what());
    return QMCRT_ERR_INVALID;
  }
}

[[noreturn]] inline void invalid(const std::string& m) { throw ApiError(QMCRT_ERR_INVALID, m); }

// Device buffer owned by the scene.
struct DBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  void alloc(size_t n) {
    if (n == bytes && p) return;
    release();
    if (n == 0) return;
    alloc_gate("cudaMalloc");
    cuda_check(cudaMalloc(&p, n), "cudaMalloc");
    bytes = n;
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

template <class T>
void upload(DBuf& b, const std::vector<T>& v) {
  b.alloc(v.size() * sizeof(T));
  if (!v.empty()) cuda_check(cudaMemcpy(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), "upload");
}

struct GridBufs {
  DBuf ranges, entries, bound, hsub, subv, sub_free, sub_cand, sub_frames;
};

class DeviceGuard {
 public:
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev_);
    if (prev_ != dev) cuda_check(cudaSetDevice(dev), "cudaSetDevice");
    switched_ = prev_ != dev;
  }
  ~DeviceGuard() {
    if (switched_) cudaSetDevice(prev_);
  }

 private:
  int prev_ = 0;
  bool switched_ = false;
};

}  // namespace qrt

struct qmcrt_scene {
  int device = 0;
  unsigned seed = 0;
  qm::SceneModel model;
  std::vector<std::unique_ptr<qrt::GridBufs>> grid_bufs;
  std::vector<qm::DevGrid> grids;
  qrt::DBuf d_grids;
  std::vector<std::unique_ptr<qrt::DBuf>> images;
  std::vector<qm::DevReceiver> receivers;
  qrt::DBuf d_receivers;
  qrt::DBuf d_local;  // focus-flat local centres then normals
  std::vector<long long> local_base;
  qrt::DBuf d_offsets;
  std::vector<long long> offset_base;
  qrt::DBuf d_samples, d_perturb;
  float sun_shape_tan = -2.0f;  // tan of the largest sun-shape angle of the local pool (-1: unbounded, -2: unknown)
  float slope_angle = -1.0f;    // largest angle of the slope-error pool from its axis, radians (< 0: unbounded)
  // walk-free flags: inputs of the last computation, device scratch
  bool flags_valid = false;
  float3 flags_sun{};
  float flags_tan = 0.f, flags_slope = 0.f;
  qrt::DBuf d_flag_tasks, d_flag_out, d_scratch_word;
  qrt::DBuf d_pool_stage;  // staging of qmcrt_set_sample_pool uploads
  qrt::DBuf d_trace_samples;  // tracer copy: d_samples in world space, P + L entries (entry i = i % P)
  qrt::DBuf d_trace_perturb;  // tracer copy of d_perturb, P + L entries
  qrt::DBuf d_offset_seg;     // heliostats + 1 starts of the per-heliostat offset segments
  int pool_size = 0;
  qrt::DBuf d_power, d_diag;
  qrt::DBuf d_chunk_power;  // per-chunk FP64 power partials of a launch (grows to the largest launch)
  qrt::DBuf d_work;         // work counter of persistent flux launches
  std::vector<qm::DevTask> templates;
  qrt::DBuf d_tasks, d_prefix;
  std::vector<int> cached_ids;
  long long cached_lights = -1;
  long long cached_chunk = -1;
  int shape = 0;  // launch shape of the production build (qmcrt_set_launch_shape)
  bool cache_valid = false;
  qm::DevTask* h_stage = nullptr;  // pinned staging for task uploads
  long long* h_prefix = nullptr;
  size_t stage_cap = 0;
  cudaEvent_t stage_done = nullptr;
  qm::SunFrame sun{};
  int exact = 0;
  int light_begin = 0, light_end = 0;
  long long total_facets = 0;

  ~qmcrt_scene() {
    if (device < 0) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    cudaDeviceSynchronize();
    if (h_stage) cudaFreeHost(h_stage);
    if (h_prefix) cudaFreeHost(h_prefix);
    if (stage_done) cudaEventDestroy(stage_done);
    grid_bufs.clear();
    images.clear();
    d_grids.release();
    d_receivers.release();
    d_local.release();
    d_offsets.release();
    d_samples.release();
    d_perturb.release();
    d_trace_samples.release();
    d_flag_tasks.release();
    d_flag_out.release();
    d_scratch_word.release();
    d_pool_stage.release();
    d_trace_perturb.release();
    d_offset_seg.release();
    d_power.release();
    d_chunk_power.release();
    d_work.release();
    d_diag.release();
    d_tasks.release();
    d_prefix.release();
    cudaSetDevice(prev);
  }
};


namespace qrt {

// Scene helpers defined in capi.cpp.
void grid_sun_data(const qm::SceneModel& m, const qm::GridModel& g, std::vector<float4>& bound,
                   std::vector<int4>& hsub, std::vector<float4>& subv);
qmcrt_scene* checked(qmcrt_scene* s);
// Sun axis and world-space tangent of the largest sun-shape angle for the
// shadow-free test (tan_local < 0: unbounded, tan_world < 0).
void sun_cone(float3 sun_dir, float tan_local, float3& axis, float& tan_world);
// out: 0 flux, 1 per-ray outcome codes, 2 bilinear deposit, 3 hit bits
// (qm::TraceOut in tracer.cu); mode: the kernel build (qmcrt_set_math_mode);
// work_counter: one device word, used by flux launches of the persistent shape.
cudaError_t launch_trace_mode(int mode, const qm::TraceParams& p, int out, cudaStream_t st, int shape = 0,
                              unsigned long long* work_counter = nullptr);
// Rays per warp chunk of the kernel a launch of (mode, shape, out) runs.
long long chunk_rays_for(int mode, int shape, int out);
// Grow-only buffer of per-chunk power partials for a launch of `chunks` warp chunks.
double* chunk_power_buffer(DBuf& buf, long long chunks);
cudaError_t run_trace(const qmcrt_scene* s, const qm::TraceParams& p, int out, cudaStream_t st,
                      unsigned long long* work_counter = nullptr);
int trace_chunk_rays();
constexpr long long kMaxTaskRays = 0x7fffffffLL - 0x10000;

}  // namespace qrt
