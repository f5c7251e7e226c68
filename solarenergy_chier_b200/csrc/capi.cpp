// C ABI (include/qmcrt.h) over the host scene model and the sm_100a kernels.
#include "qmcrt.h"
#include "helio_geom.h"
#include "prep.h"
#include "grid_build.h"
#include "power.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "device_scene.h"
#include "pools.h"
#include "sampling.h"
#include "scene.h"
#include "smooth.h"
#include "tracer.h"
#include "vecmath.h"
#include "runtime.h"

namespace {
thread_local std::string g_last_error;

// Allocations left before an injected failure (< 0: injection off).
std::atomic<long long> g_fail_after{[] {
  const char* v = std::getenv("QMCRT_INJECT_ALLOC_FAILURE");
  return v && *v ? std::atoll(v) : -1LL;
}()};
}  // namespace

namespace qm {
void set_last_error(const std::string& msg) { g_last_error = msg; }
}  // namespace qm

using namespace qrt;

namespace qrt {

void alloc_gate(const char* what) {
  long long left = g_fail_after.load();
  while (left >= 0 && !g_fail_after.compare_exchange_weak(left, left - 1)) {
  }
  if (left == 0) throw ApiError(QMCRT_ERR_NOMEM, std::string(what) + ": injected allocation failure");
}

using qm::DevGrid;
using qm::DevReceiver;
using qm::DevTask;

// Sun-dependent data of one grid: per heliostat its traversal record and
// (first sub-heliostat, count, lattice rows, lattice columns), and per
// sub-heliostat its parallelogram as A, B - A, C - A.
void grid_sun_data(const qm::SceneModel& m, const qm::GridModel& g, std::vector<float4>& bound,
                   std::vector<int4>& hsub, std::vector<float4>& subv) {
  bound.assign(5 * (size_t)g.num_heliostats, float4{});
  hsub.assign(g.num_heliostats, int4{});
  for (int i = 0; i < g.num_heliostats; ++i) {
    const qm::HeliostatModel& h = m.heliostats[g.start_heliostat + i];
    int2 rc;
    qm::heliostat_record(g.sub_vertices.data() + 3 * (size_t)h.sub_begin, h.num_sub, h.row_col, h.pos, h.normal,
                         &bound[5 * (size_t)i], &rc);
    hsub[i] = make_int4(h.sub_begin, h.num_sub, rc.x, rc.y);
  }
  subv.assign(3 * (size_t)g.num_subheliostats, float4{});
  for (int sidx = 0; sidx < g.num_subheliostats; ++sidx) {
    const float3 B = g.sub_vertices[3 * sidx], A = g.sub_vertices[3 * sidx + 1], C = g.sub_vertices[3 * sidx + 2];
    const float3 ab = qm::sub(B, A), ac = qm::sub(C, A);
    subv[3 * sidx] = make_float4(A.x, A.y, A.z, ab.x);
    subv[3 * sidx + 1] = make_float4(ab.y, ab.z, ac.x, ac.y);
    subv[3 * sidx + 2] = make_float4(ac.z, 0.f, 0.f, 0.f);
  }
}

// Sun frame and per-heliostat task templates (both depend on the sun).
void build_templates(qmcrt_scene* s) {
  const qm::SceneModel& m = s->model;
  const qm::SceneConfig& cfg = m.config;
  // Sun frame of -sun_dir (QuasiMonteCarloRayTracer::generateSunrayArgument feeds
  // -sunray_direction to local2world_rotate per ray; the frame is constant).
  qm::Frame f = qm::make_frame(qm::neg(cfg.sun_dir), false);
  s->sun.u = f.u;
  s->sun.n = f.n;
  s->sun.v = f.v;
  s->sun.identity = f.identity ? 1 : 0;

  s->templates.assign(m.heliostats.size(), DevTask{});
  for (size_t i = 0; i < m.heliostats.size(); ++i) {
    const auto& h = m.heliostats[i];
    const auto& g = m.grids[h.grid];
    const auto& r = m.receivers[g.receiver];
    DevTask t{};
    t.type = h.type;
    t.grid = h.grid;
    t.receiver = g.receiver;
    t.own = (int)i - g.start_heliostat;
    t.num_facets = h.num_facets;
    t.power_slot = (int)i;
    t.row_col = h.row_col;
    t.sub_row_col = h.sub_row_col;
    t.pixel_length = h.pixel_length;
    // QuasiMonteCarloRayTracer::rayTracing (QuasiMonteCarloRayTracer.cpp:58-60).
    float ratio = h.pixel_length / r.pixel_length;
    t.factor = cfg.dni * ratio * ratio * cfg.helio_reflected_rate / float(cfg.num_per_sunshape_group);
    t.gap = h.gap;
    t.sub_length = h.sub_length;
    t.size = h.size;
    t.pos = h.pos;
    t.normal = h.normal;
    qm::Frame hf = qm::make_frame(h.normal, h.type == 1);
    t.fu = hf.u;
    t.fn = hf.n;
    t.fv = hf.v;
    t.frame_identity = hf.identity ? 1 : 0;
    if (h.type == 1) {
      const float3* base = s->d_local.as<float3>() + s->local_base[i];
      t.local_centers = base;
      t.local_normals = base + h.local_centers.size();
    }
    t.offsets = s->d_offsets.as<int>() + s->offset_base[i];
    t.samples = s->d_trace_samples.as<float4>();
    t.perturbations = s->d_trace_perturb.as<float4>();
    t.pool_size = s->pool_size;
    s->templates[i] = t;
  }
  s->cache_valid = false;
}

void build_device_scene(qmcrt_scene* s) {
  qm::SceneModel& m = s->model;
  const qm::SceneConfig& cfg = m.config;
  if (cfg.num_sunshape_groups <= 0 || cfg.num_per_sunshape_group <= 0) invalid("sun-shape pool size must be positive");
  long long P = (long long)cfg.num_sunshape_groups * cfg.num_per_sunshape_group;
  if (P > (1LL << 30)) invalid("sun-shape pool is larger than 2^30 samples");
  s->pool_size = (int)P;
  s->light_begin = 0;
  s->light_end = cfg.num_per_sunshape_group;

  // Grids.
  s->grid_bufs.clear();
  s->grids.clear();
  for (auto& g : m.grids) {
    auto gb = std::make_unique<GridBufs>();
    // Cell lists in traversal form: a [begin, end) pair per cell and, per
    // entry, the heliostat with its sub-heliostat range inline.
    std::vector<int2> ranges(g.cell_hindex.size() > 0 ? g.cell_hindex.size() - 1 : 0);
    for (size_t c = 0; c < ranges.size(); ++c) ranges[c] = make_int2(g.cell_hindex[c], g.cell_hindex[c + 1]);
    std::vector<int4> entries(g.cell_hmatch.size());
    for (size_t k = 0; k < entries.size(); ++k) {
      const qm::HeliostatModel& h = m.heliostats[g.start_heliostat + g.cell_hmatch[k]];
      entries[k] = make_int4(g.cell_hmatch[k], h.sub_begin, h.num_sub, 0);
    }
    upload(gb->ranges, ranges);
    upload(gb->entries, entries);
    std::vector<float4> bound, subv;
    std::vector<int4> hsub;
    grid_sun_data(m, g, bound, hsub, subv);
    upload(gb->bound, bound);
    upload(gb->hsub, hsub);
    upload(gb->subv, subv);
    // block-free flags start cleared (no skipping) until the pools exist
    upload(gb->sub_free, std::vector<int>(std::max(g.num_subheliostats, 1), 0));
    upload(gb->sub_cand, std::vector<int>((size_t)std::max(g.num_subheliostats, 1) * qm::kMaxCandidates, -1));
    gb->sub_frames.alloc((size_t)std::max(g.num_subheliostats, 1) * 6 * sizeof(float4));
    cuda_check(cudaMemset(gb->sub_frames.p, 0, gb->sub_frames.bytes), "cudaMemset");
    DevGrid dg;
    dg.pos = g.pos;
    dg.interval = g.interval;
    dg.cells = g.cells;
    dg.max_steps = g.cells.x + g.cells.y + g.cells.z + 2;
    dg.cell_range = gb->ranges.as<int2>();
    dg.entries = gb->entries.as<int4>();
    dg.bound = gb->bound.as<float4>();
    dg.hsub = gb->hsub.as<int4>();
    dg.subv = gb->subv.as<float4>();
    dg.sub_free = gb->sub_free.as<int>();
    dg.sub_cand = gb->sub_cand.as<int>();
    dg.sub_frames = gb->sub_frames.as<float4>();
    s->grids.push_back(dg);
    s->grid_bufs.push_back(std::move(gb));
  }
  upload(s->d_grids, s->grids);

  // Receivers and images.
  s->images.clear();
  s->receivers.clear();
  for (auto& r : m.receivers) {
    auto img = std::make_unique<DBuf>();
    size_t n = (size_t)std::max(r.resolution.x, 0) * std::max(r.resolution.y, 0);
    img->alloc(std::max<size_t>(n, 1) * sizeof(float));
    cuda_check(cudaMemset(img->p, 0, img->bytes), "cudaMemset");
    DevReceiver dr{};
    dr.type = r.type;
    dr.resolution = r.resolution;
    dr.image = img->as<float>();
    if (r.type == 0) {
      dr.a = r.vertex[0];
      dr.ab = qm::sub(r.vertex[1], r.vertex[0]);
      dr.ac = qm::sub(r.vertex[3], r.vertex[0]);
    }
    dr.pos = r.pos;
    dr.size = r.size;
    // the loader refuses empty images, so the height lies in [1/ppm, 2^31/ppm]
    // and its reciprocal is a normal float
    dr.rcp_height = r.type == 1 ? 1.0f / r.size.y : 0.0f;
    s->receivers.push_back(dr);
    s->images.push_back(std::move(img));
  }
  upload(s->d_receivers, s->receivers);

  // Focus-flat local facet frames.
  std::vector<float3> local;
  s->local_base.assign(m.heliostats.size(), -1);
  for (size_t i = 0; i < m.heliostats.size(); ++i) {
    const auto& h = m.heliostats[i];
    if (h.type != 1) continue;
    s->local_base[i] = (long long)local.size();
    local.insert(local.end(), h.local_centers.begin(), h.local_centers.end());
    local.insert(local.end(), h.local_normals.begin(), h.local_normals.end());
  }
  upload(s->d_local, local);

  // Pool offsets: num_facets + 1 per heliostat in one buffer.
  s->offset_base.assign(m.heliostats.size(), 0);
  long long total = 0;
  s->total_facets = 0;
  for (size_t i = 0; i < m.heliostats.size(); ++i) {
    s->offset_base[i] = total;
    total += (long long)m.heliostats[i].num_facets + 1;
    s->total_facets += m.heliostats[i].num_facets;
  }
  s->d_offsets.alloc((size_t)total * sizeof(int));

  s->d_samples.alloc((size_t)P * sizeof(float4));
  s->d_perturb.alloc((size_t)P * sizeof(float4));
  s->d_trace_samples.alloc((size_t)(P + cfg.num_per_sunshape_group) * sizeof(float4));
  s->d_scratch_word.alloc(sizeof(unsigned));
  s->d_trace_perturb.alloc((size_t)(P + cfg.num_per_sunshape_group) * sizeof(float4));
  {
    std::vector<long long> seg(s->offset_base);
    seg.push_back(total);
    upload(s->d_offset_seg, seg);
  }
  s->d_power.alloc(std::max<size_t>(m.heliostats.size(), 1) * sizeof(double));
  cuda_check(cudaMemset(s->d_power.p, 0, s->d_power.bytes), "cudaMemset");
  s->d_diag.alloc(qm::kDiagSlots * sizeof(unsigned long long));
  cuda_check(cudaMemset(s->d_diag.p, 0, s->d_diag.bytes), "cudaMemset");

  build_templates(s);
  s->cache_valid = false;
}

void generate_offsets(qmcrt_scene* s, unsigned seed) {
  const long long total = (long long)(s->d_offsets.bytes / sizeof(int));
  cuda_check(qm::launch_offsets_all(s->d_offsets.as<int>(), s->d_offset_seg.as<long long>(),
                                    (int)s->model.heliostats.size(), total, seed, s->pool_size, 0),
             "offsets kernel");
  cuda_check(cudaDeviceSynchronize(), "offsets kernel");
}

// Sun axis and tangent of the largest sun-shape angle in world space, for
// the shadow-free test, from the tangent `tan_local` of the local pool (the
// sun frame maps the local y axis to -sun_dir, which may not be unit length;
// an identity frame leaves samples as they are).
void sun_cone(float3 sun_dir, float tan_local, float3& axis, float& tan_world) {
  const qm::Frame f = qm::make_frame(qm::neg(sun_dir), false);
  if (f.identity) {
    axis = make_float3(0.f, 1.f, 0.f);
    tan_world = tan_local;
    return;
  }
  axis = qm::neg(sun_dir);
  const double len = std::sqrt((double)sun_dir.x * sun_dir.x + (double)sun_dir.y * sun_dir.y +
                               (double)sun_dir.z * sun_dir.z);
  tan_world = tan_local < 0.0f ? -1.0f : (float)(tan_local / len);
}

// Tangent of the largest angle between a pool direction and the pool's
// local +y axis, reduced on the device (-1 when some direction has y <= 0:
// unbounded).
float pool_tan(qmcrt_scene* s, const DBuf& pool) {
  cuda_check(cudaMemset(s->d_scratch_word.p, 0, sizeof(unsigned)), "cudaMemset");
  cuda_check(qm::launch_pool_tan(pool.as<float4>(), s->pool_size, s->d_scratch_word.as<unsigned>(), 0), "pool bound");
  unsigned bits = 0;
  cuda_check(cudaMemcpy(&bits, s->d_scratch_word.p, sizeof(unsigned), cudaMemcpyDeviceToHost), "pool bound");
  float t;
  std::memcpy(&t, &bits, sizeof(t));
  return std::isfinite(t) ? t : -1.0f;
}

// Walk-free flags (csrc/shadow.h) for the current sun and pools, computed on
// the device: per heliostat template for the shadow walks, per sub-heliostat
// (each grid's sub_free array) for the block walks.  Skipped when neither the
// sun nor the pools' angular bounds changed since the last computation.
void update_shadow_flags(qmcrt_scene* s, bool pools_changed) {
  if (pools_changed || s->sun_shape_tan < -1.5f) {
    s->sun_shape_tan = pool_tan(s, s->d_samples);
    const float slope_tan = pool_tan(s, s->d_perturb);
    s->slope_angle = slope_tan < 0.0f ? -1.0f : std::atan(slope_tan);
  }
  const float3 sun = s->model.config.sun_dir;
  if (s->flags_valid && sun.x == s->flags_sun.x && sun.y == s->flags_sun.y && sun.z == s->flags_sun.z &&
      s->sun_shape_tan == s->flags_tan && s->slope_angle == s->flags_slope)
    return;
  float3 axis;
  float tan_world;
  sun_cone(sun, s->sun_shape_tan, axis, tan_world);
  qm::WalkFlagParams p{};
  upload(s->d_flag_tasks, s->templates);
  s->d_flag_out.alloc(std::max<size_t>(s->templates.size(), 1) * (1 + qm::kMaxCandidates) * sizeof(int));
  p.tasks = s->d_flag_tasks.as<DevTask>();
  p.n = (int)s->templates.size();
  p.max_sub = 0;
  for (const auto& h : s->model.heliostats) p.max_sub = std::max(p.max_sub, h.num_sub);
  p.grids = s->d_grids.as<DevGrid>();
  p.sun_axis = axis;
  p.sun_tan = tan_world;
  p.sun_dir = sun;
  p.block_theta = tan_world < 0.0f || s->slope_angle < 0.0f ? -1.0f : std::atan(tan_world) + 2.0f * s->slope_angle;
  const size_t nt = s->templates.size();
  p.shadow_out = s->d_flag_out.as<int>();
  p.shadow_cand_out = s->d_flag_out.as<int>() + nt;
  cuda_check(qm::launch_walk_flags(p, 0), "walk flags");
  std::vector<int> flags(nt * (1 + qm::kMaxCandidates));
  if (!flags.empty())
    cuda_check(cudaMemcpy(flags.data(), s->d_flag_out.p, flags.size() * sizeof(int), cudaMemcpyDeviceToHost),
               "walk flags");
  for (size_t i = 0; i < nt; ++i) {
    s->templates[i].shadow_free = flags[i];
    for (int k = 0; k < qm::kMaxCandidates; ++k)
      s->templates[i].shadow_cand[k] = flags[nt + i * qm::kMaxCandidates + k];
  }
  s->flags_valid = true;
  s->flags_sun = sun;
  s->flags_tan = s->sun_shape_tan;
  s->flags_slope = s->slope_angle;
  s->cache_valid = false;
}

// The tracer's copies of the pools (world-space samples, P + L entries);
// redone after every change of the pools or of the sun, with the
// shadow-free flags that depend on both.
void rotate_pool(qmcrt_scene* s, bool pools_changed) {
  const int n_out = s->pool_size + s->model.config.num_per_sunshape_group;
  cuda_check(qm::launch_trace_pools(s->d_samples.as<float4>(), s->d_perturb.as<float4>(), s->pool_size, n_out, s->sun,
                                    s->d_trace_samples.as<float4>(), s->d_trace_perturb.as<float4>(), 0),
             "pool rotation");
  cuda_check(cudaDeviceSynchronize(), "pool rotation");
  update_shadow_flags(s, pools_changed);
}

void generate_pool(qmcrt_scene* s, unsigned seed, int sunshape, float half_angle) {
  const qm::SceneConfig& cfg = s->model.config;
  qm::PoolParams p{};
  p.samples = s->d_samples.as<float4>();
  p.perturbations = s->d_perturb.as<float4>();
  p.pool_size = s->pool_size;
  p.sunshape = sunshape;
  p.half_angle = half_angle;
  p.sigma = cfg.helio_disturb_std;
  p.seed_sun = qm::mix32(seed * 2654435761u + 1u);
  p.seed_slope = qm::mix32(seed * 2654435761u + 2u);
  DBuf cdf, kk;
  if (sunshape == qm::kSunshapeBuie) {
    if (cfg.inverse_transform_sampling_groups <= 0) invalid("inverse_transform_sampling_groups must be positive");
    qm::BuieHost t = qm::build_buie_table(cfg.csr, cfg.inverse_transform_sampling_groups);
    upload(cdf, t.cdf);
    upload(kk, t.k);
    p.buie.cdf = cdf.as<float2>();
    p.buie.k = kk.as<float>();
    p.buie.n = cfg.inverse_transform_sampling_groups;
    p.buie.less_465 = t.less_465;
    p.buie.gamma = t.gamma;
    p.buie.A = t.A;
    p.buie.B = t.B;
    p.buie.C = t.C;
  } else if (sunshape != qm::kSunshapePillbox) {
    invalid("sunshape must be 0 (Buie) or 1 (pillbox)");
  }
  cuda_check(qm::launch_pool(p, 0), "pool kernel");
  cuda_check(cudaDeviceSynchronize(), "pool kernel");
  rotate_pool(s, true);
}

qmcrt_scene* checked(qmcrt_scene* s) {
  if (!s) invalid("scene is NULL");
  if (s->device < 0) throw ApiError(QMCRT_ERR_STATE, "scene was loaded host-only (device -1); it cannot trace");
  return s;
}

void check_heliostat(const qmcrt_scene* s, int id) {
  // QuasiMonteCarloRayTracer::checkValidHeliostatIndex (QuasiMonteCarloRayTracer.cpp:96-127).
  int n = (int)s->model.heliostats.size();
  if (id < 0 || id >= n)
    invalid("The ray tracing heliostat index " + std::to_string(id) +
            " is invalid. The heliostat index should between 0 and " + std::to_string(n) + ".");
}

void ensure_stage(qmcrt_scene* s, size_t n) {
  if (s->stage_done) cuda_check(cudaEventSynchronize(s->stage_done), "cudaEventSynchronize");
  if (n <= s->stage_cap) return;
  if (s->h_stage) cudaFreeHost(s->h_stage);
  if (s->h_prefix) cudaFreeHost(s->h_prefix);
  s->h_stage = nullptr;
  s->h_prefix = nullptr;
  size_t cap = std::max<size_t>(n, 64);
  alloc_gate("cudaMallocHost");
  cuda_check(cudaMallocHost((void**)&s->h_stage, cap * sizeof(DevTask)), "cudaMallocHost");
  alloc_gate("cudaMallocHost");
  cuda_check(cudaMallocHost((void**)&s->h_prefix, (cap + 1) * sizeof(long long)), "cudaMallocHost");
  s->d_tasks.alloc(cap * sizeof(DevTask));
  s->d_prefix.alloc((cap + 1) * sizeof(long long));
  s->stage_cap = cap;
  s->cache_valid = false;
}

qm::TraceParams base_params(qmcrt_scene* s) {
  qm::TraceParams p{};
  p.grids = s->d_grids.as<DevGrid>();
  p.receivers = s->d_receivers.as<DevReceiver>();
  p.light_begin = s->light_begin;
  p.light_end = s->light_end;
  p.power = s->d_power.as<double>();
  p.diag = s->d_diag.as<unsigned long long>();
  return p;
}

// Launch shapes of the production build (math mode 0) that the autotuner
// times: threads per block and warp-chunk iterations, all at 72 registers
// except the 256-thread shape (64 registers, as math mode 2), and a
// persistent shape (resident warps taking chunks from a work counter).  A shape
// changes how rays are handed to warps, never a ray's arithmetic.  Shapes
// other than 0 serve flux launches only; records, hit bits and bilinear
// deposits keep shape 0, whose chunk layout the other outputs share.
struct LaunchShape {
  int threads, chunk_iters, persistent;
  cudaError_t (*launch)(const qm::TraceParams&, int, cudaStream_t, unsigned long long*);
  int (*chunk_rays)();
};
const LaunchShape kShapes[] = {
    {32, 64, 0, qm::launch_trace_fast, qm::trace_chunk_rays_fast},
    {32, 32, 0, qm::launch_trace_fast_c32, qm::trace_chunk_rays_fast_c32},
    {32, 128, 0, qm::launch_trace_fast_c128, qm::trace_chunk_rays_fast_c128},
    {64, 64, 0, qm::launch_trace_fast_t64, qm::trace_chunk_rays_fast_t64},
    {256, 64, 0, qm::launch_trace_fast4, qm::trace_chunk_rays_fast4},
    {32, 64, 1, qm::launch_trace_fast_ps, qm::trace_chunk_rays_fast_ps},
};
constexpr int kNumShapes = sizeof(kShapes) / sizeof(kShapes[0]);

int shape_for(int mode, int shape, int out) { return (mode == 0 && out == 0 && shape > 0 && shape < kNumShapes) ? shape : 0; }

long long chunk_rays_for(int mode, int shape, int out) {
  return kShapes[shape_for(mode, shape, out)].chunk_rays();
}

cudaError_t launch_trace_mode(int mode, const qm::TraceParams& p, int out, cudaStream_t st, int shape,
                              unsigned long long* work_counter) {
  cudaError_t e;
  switch (mode) {
    case 1: e = qm::launch_trace_exact(p, out, st); break;
    case 2: e = qm::launch_trace_fast4(p, out, st); break;
    case 3: e = qm::launch_trace_approx(p, out, st); break;
    case 4: e = qm::launch_trace_rx(p, out, st); break;
    default: e = kShapes[shape_for(mode, shape, out)].launch(p, out, st, work_counter); break;
  }
  // flux and bilinear-deposit launches add their per-chunk power partials
  if (e == cudaSuccess && (out == 0 || out == 2) && p.chunk_power) e = qm::launch_power_reduce(p, st);
  return e;
}

double* chunk_power_buffer(DBuf& buf, long long chunks) {
  const size_t need = (size_t)std::max<long long>(chunks, 1) * sizeof(double);
  if (buf.bytes < need) buf.alloc(need);
  return buf.as<double>();
}

cudaError_t run_trace(const qmcrt_scene* s, const qm::TraceParams& p, int out, cudaStream_t st,
                      unsigned long long* work_counter) {
  return launch_trace_mode(s->exact, p, out, st, s->shape, work_counter);
}

// Traces heliostats ids[0..n) over the scene's light range: out 0 adds their
// flux and FP64 power, out 3 writes one hit bit per ray into hit_bits
// (one 32-bit word per warp iteration of every warp chunk, chunks in task
// order) and nothing else.  Returns the launch's number of warp chunks.
long long trace_ids(qmcrt_scene* s, const int* ids, int n, cudaStream_t stream, int out = 0,
                    uint32_t* hit_bits = nullptr) {
  if (n < 0 || (n > 0 && !ids)) invalid("heliostat list is invalid");
  for (int i = 0; i < n; ++i) check_heliostat(s, ids[i]);
  if (n == 0) return 0;
  for (int i = 0; i < n; ++i)
    if ((long long)s->templates[ids[i]].num_facets * (s->light_end - s->light_begin) > kMaxTaskRays)
      invalid("a heliostat's micro-facets x lights must stay below 2^31 - 2^16 rays per launch; trace fewer lights");
  DeviceGuard guard(s->device);
  const long long nl = s->light_end - s->light_begin;
  if (nl == 0) return 0;
  const long long chunk = chunk_rays_for(s->exact, s->shape, out);
  auto chunks_of = [&](int id) { return ((long long)s->templates[id].num_facets * nl + chunk - 1) / chunk; };
  bool same = s->cache_valid && s->cached_lights == nl && s->cached_chunk == chunk && (int)s->cached_ids.size() == n &&
              std::equal(ids, ids + n, s->cached_ids.begin());
  long long total = 0;
  if (!same) {
    ensure_stage(s, (size_t)n);
    s->h_prefix[0] = 0;
    for (int i = 0; i < n; ++i) {
      s->h_stage[i] = s->templates[ids[i]];
      s->h_prefix[i + 1] = s->h_prefix[i] + chunks_of(ids[i]);
    }
    cuda_check(cudaMemcpyAsync(s->d_tasks.p, s->h_stage, n * sizeof(DevTask), cudaMemcpyHostToDevice, stream),
               "task upload");
    cuda_check(cudaMemcpyAsync(s->d_prefix.p, s->h_prefix, (n + 1) * sizeof(long long), cudaMemcpyHostToDevice, stream),
               "task upload");
    if (!s->stage_done) cuda_check(cudaEventCreateWithFlags(&s->stage_done, cudaEventDisableTiming), "cudaEventCreate");
    cuda_check(cudaEventRecord(s->stage_done, stream), "cudaEventRecord");
    s->cached_ids.assign(ids, ids + n);
    s->cached_lights = nl;
    s->cached_chunk = chunk;
    s->cache_valid = true;
  }
  for (int i = 0; i < n; ++i) total += chunks_of(ids[i]);
  qm::TraceParams p = base_params(s);
  p.tasks = s->d_tasks.as<DevTask>();
  p.facet_prefix = s->d_prefix.as<long long>();
  p.num_tasks = n;
  p.total_facets = total;
  p.hit_bits = hit_bits;
  if (out == 3 && !hit_bits) return total;
  unsigned long long* work = nullptr;
  if (out == 0) {
    p.chunk_power = chunk_power_buffer(s->d_chunk_power, total);
    if (s->d_work.bytes < sizeof(unsigned long long)) s->d_work.alloc(sizeof(unsigned long long));
    work = s->d_work.as<unsigned long long>();
  }
  cuda_check(run_trace(s, p, out, stream, work), "trace kernel");
  return total;
}

int trace_chunk_rays() { return qm::trace_chunk_rays_fast(); }

}  // namespace qrt

extern "C" {

const char* qmcrt_last_error(void) { return g_last_error.c_str(); }

int qmcrt_debug_fail_allocations(long long after) {
  g_fail_after.store(after < 0 ? -1 : after);
  return QMCRT_OK;
}

int qmcrt_version(void) { return 1; }

int qmcrt_scene_load(const char* scene_path, const char* config_path, int device, unsigned seed, qmcrt_scene** out) {
  return guarded([&] {
    if (!out) invalid("out is NULL");
    *out = nullptr;
    if (!scene_path || !config_path) invalid("scene and configuration paths are required");
    if (device >= 0) {
      int ndev = 0;
      cuda_check(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
      if (device >= ndev) invalid("device index out of range");
    }
    alloc_gate("scene state");
    std::unique_ptr<qmcrt_scene> s(new qmcrt_scene());
    s->device = device;
    s->seed = seed;
    std::string err;
    int fields = qm::read_config_file(config_path, s->model.config, err);
    if (fields < 0) throw ApiError(QMCRT_ERR_IO, err);
    qm::SceneConfig cfg = s->model.config;
    if (!qm::read_scene_file(scene_path, s->model, err)) throw ApiError(QMCRT_ERR_IO, err);
    s->model.config = cfg;
    s->model.config_fields = fields;
    if (!qm::process_scene(s->model, err)) throw ApiError(QMCRT_ERR_INVALID, err);
    if (device < 0) {
      // Host-only scene: the processed model without device buffers, for
      // inspecting geometry on a machine without a GPU.
      const auto& c = s->model.config;
      s->pool_size = c.num_sunshape_groups * c.num_per_sunshape_group;
      for (const auto& h : s->model.heliostats) s->total_facets += h.num_facets;
      *out = s.release();
      return;
    }
    DeviceGuard guard(device);
    build_device_scene(s.get());
    generate_pool(s.get(), seed, qm::kSunshapeBuie, 0.00465f);
    generate_offsets(s.get(), seed);
    *out = s.release();
  });
}

void qmcrt_scene_free(qmcrt_scene* s) { delete s; }

int qmcrt_config_check(const char* config_path, int* fields) {
  return guarded([&] {
    if (!config_path) invalid("configuration path is NULL");
    qm::SceneConfig cfg;
    std::string err;
    const int n = qm::read_config_file(config_path, cfg, err);
    if (n < 0) throw ApiError(QMCRT_ERR_IO, err);
    if (fields) *fields = n;
  });
}

int qmcrt_scene_get_info(const qmcrt_scene* s, qmcrt_scene_info* info) {
  return guarded([&] {
    if (!s || !info) invalid("scene or info is NULL");
    const auto& m = s->model;
    const auto& c = m.config;
    std::memset(info, 0, sizeof(*info));
    info->num_receivers = (int)m.receivers.size();
    info->num_grids = (int)m.grids.size();
    info->num_heliostats = (int)m.heliostats.size();
    info->num_sunshape_groups = c.num_sunshape_groups;
    info->num_per_sunshape_group = c.num_per_sunshape_group;
    info->pool_size = s->pool_size;
    info->inverse_transform_sampling_groups = c.inverse_transform_sampling_groups;
    info->config_fields = m.config_fields;
    info->sun_dir[0] = c.sun_dir.x;
    info->sun_dir[1] = c.sun_dir.y;
    info->sun_dir[2] = c.sun_dir.z;
    info->dni = c.dni;
    info->csr = c.csr;
    info->receiver_pixel_length = c.receiver_pixel_length;
    info->helio_disturb_std = c.helio_disturb_std;
    info->helio_pixel_length = c.helio_pixel_length;
    info->helio_reflected_rate = c.helio_reflected_rate;
    info->ground_length = m.ground_length;
    info->ground_width = m.ground_width;
    info->total_facets = s->total_facets;
  });
}

int qmcrt_receiver_get(const qmcrt_scene* s, int id, int* type, int* width, int* height, float* pixel_length,
                       float* vertices12, float* normal3, float* focus3) {
  return guarded([&] {
    if (!s) invalid("scene is NULL");
    if (id < 0 || id >= (int)s->model.receivers.size()) invalid("receiver index out of range");
    const auto& r = s->model.receivers[id];
    if (type) *type = r.type;
    if (width) *width = r.resolution.x;
    if (height) *height = r.resolution.y;
    if (pixel_length) *pixel_length = r.pixel_length;
    if (vertices12)
      for (int k = 0; k < 4; ++k) {
        vertices12[3 * k] = r.vertex[k].x;
        vertices12[3 * k + 1] = r.vertex[k].y;
        vertices12[3 * k + 2] = r.vertex[k].z;
      }
    if (normal3) {
      normal3[0] = r.normal.x;
      normal3[1] = r.normal.y;
      normal3[2] = r.normal.z;
    }
    if (focus3) {
      focus3[0] = r.focus.x;
      focus3[1] = r.focus.y;
      focus3[2] = r.focus.z;
    }
  });
}

int qmcrt_heliostat_get(const qmcrt_scene* s, int id, int* type, int* grid, int* num_facets, int* num_sub,
                        int* sub_begin, float* pos3, float* size3, float* normal3, float* focus_length) {
  return guarded([&] {
    if (!s) invalid("scene is NULL");
    check_heliostat(s, id);
    const auto& h = s->model.heliostats[id];
    if (type) *type = h.type;
    if (grid) *grid = h.grid;
    if (num_facets) *num_facets = h.num_facets;
    if (num_sub) *num_sub = h.num_sub;
    if (sub_begin) *sub_begin = h.sub_begin;
    if (pos3) pos3[0] = h.pos.x, pos3[1] = h.pos.y, pos3[2] = h.pos.z;
    if (size3) size3[0] = h.size.x, size3[1] = h.size.y, size3[2] = h.size.z;
    if (normal3) normal3[0] = h.normal.x, normal3[1] = h.normal.y, normal3[2] = h.normal.z;
    if (focus_length) *focus_length = h.focus_length;
  });
}

int qmcrt_grid_get(const qmcrt_scene* s, int id, int* cells3, int* num_sub, int* nnz, int* receiver, int* start,
                   int* count) {
  return guarded([&] {
    if (!s) invalid("scene is NULL");
    if (id < 0 || id >= (int)s->model.grids.size()) invalid("grid index out of range");
    const auto& g = s->model.grids[id];
    if (cells3) cells3[0] = g.cells.x, cells3[1] = g.cells.y, cells3[2] = g.cells.z;
    if (num_sub) *num_sub = g.num_subheliostats;
    if (nnz) *nnz = (int)g.cell_match.size();
    if (receiver) *receiver = g.receiver;
    if (start) *start = g.start_heliostat;
    if (count) *count = g.num_heliostats;
  });
}

int qmcrt_grid_csr(const qmcrt_scene* s, int id, int* index, int* match) {
  return guarded([&] {
    if (!s) invalid("scene is NULL");
    if (id < 0 || id >= (int)s->model.grids.size()) invalid("grid index out of range");
    const auto& g = s->model.grids[id];
    if (index) std::copy(g.cell_index.begin(), g.cell_index.end(), index);
    if (match) std::copy(g.cell_match.begin(), g.cell_match.end(), match);
  });
}

int qmcrt_grid_vertices(const qmcrt_scene* s, int id, float* xyz) {
  return guarded([&] {
    if (!s || !xyz) invalid("scene or output is NULL");
    if (id < 0 || id >= (int)s->model.grids.size()) invalid("grid index out of range");
    const auto& g = s->model.grids[id];
    for (size_t i = 0; i < g.sub_vertices.size(); ++i) {
      xyz[3 * i] = g.sub_vertices[i].x;
      xyz[3 * i + 1] = g.sub_vertices[i].y;
      xyz[3 * i + 2] = g.sub_vertices[i].z;
    }
  });
}

int qmcrt_heliostat_facets(qmcrt_scene* s, int id, float* origins, float* normals) {
  return guarded([&] {
    checked(s);
    check_heliostat(s, id);
    if (!origins || !normals) invalid("output is NULL");
    DeviceGuard guard(s->device);
    const DevTask& t = s->templates[id];
    DBuf o, n;
    o.alloc(std::max<size_t>(t.num_facets, 1) * sizeof(float3));
    n.alloc(std::max<size_t>(t.num_facets, 1) * sizeof(float3));
    cudaError_t e = s->exact == 1 ? qm::launch_facets_exact(t, o.as<float3>(), n.as<float3>(), 0)
                                  : qm::launch_facets_fast(t, o.as<float3>(), n.as<float3>(), 0);
    cuda_check(e, "facets kernel");
    cuda_check(cudaMemcpy(origins, o.p, (size_t)t.num_facets * sizeof(float3), cudaMemcpyDeviceToHost), "readback");
    cuda_check(cudaMemcpy(normals, n.p, (size_t)t.num_facets * sizeof(float3), cudaMemcpyDeviceToHost), "readback");
  });
}

int qmcrt_scene_set_sun(qmcrt_scene* s, const float* sun_dir) {
  return guarded([&] {
    if (!s) invalid("scene is NULL");
    if (!sun_dir) invalid("sun direction is NULL");
    const float3 d = make_float3(sun_dir[0], sun_dir[1], sun_dir[2]);
    if (!std::isfinite(d.x) || !std::isfinite(d.y) || !std::isfinite(d.z) || (d.x == 0 && d.y == 0 && d.z == 0))
      invalid("sun direction must be finite and non-zero");
    qm::set_sun(s->model, d);
    if (s->device < 0) return;
    DeviceGuard guard(s->device);
    cuda_check(cudaDeviceSynchronize(), "set_sun");
    for (size_t g = 0; g < s->model.grids.size(); ++g) {
      std::vector<float4> bound, subv;
      std::vector<int4> hsub;
      grid_sun_data(s->model, s->model.grids[g], bound, hsub, subv);
      upload(s->grid_bufs[g]->bound, bound);
      upload(s->grid_bufs[g]->hsub, hsub);
      upload(s->grid_bufs[g]->subv, subv);
      s->grids[g].bound = s->grid_bufs[g]->bound.as<float4>();
      s->grids[g].hsub = s->grid_bufs[g]->hsub.as<int4>();
      s->grids[g].subv = s->grid_bufs[g]->subv.as<float4>();
    }
    upload(s->d_grids, s->grids);
    build_templates(s);
    s->flags_valid = false;
    rotate_pool(s, false);
  });
}

int qmcrt_set_sample_pool(qmcrt_scene* s, const float* dirs, const float* perturb, int groups, int per_group,
                          int on_device) {
  return guarded([&] {
    checked(s);
    if (!dirs || !perturb) invalid("pool pointers are NULL");
    if (groups <= 0 || per_group <= 0 || (long long)groups * per_group != s->pool_size ||
        per_group != s->model.config.num_per_sunshape_group)
      invalid("pool shape must match the configuration's groups x lights-per-group");
    DeviceGuard guard(s->device);
    const int n = s->pool_size;
    // staging for both xyz pools and a counter word after them, kept with the
    // scene (allocated once)
    DBuf& tmp = s->d_pool_stage;
    const size_t stage_bytes = (size_t)n * 6 * sizeof(float) + sizeof(unsigned);
    if (tmp.bytes < stage_bytes) tmp.alloc(stage_bytes);
    float* stage_dirs = tmp.as<float>();
    float* stage_pert = stage_dirs + (size_t)n * 3;
    unsigned* bad = reinterpret_cast<unsigned*>(stage_pert + (size_t)n * 3);
    const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    cuda_check(cudaMemcpy(stage_dirs, dirs, (size_t)n * 3 * sizeof(float), kind), "pool upload");
    cuda_check(cudaMemcpy(stage_pert, perturb, (size_t)n * 3 * sizeof(float), kind), "pool upload");
    // Both pools must hold unit vectors (the tracer normalises the perturbed
    // normal and the reflected ray without a range test); the scene's pools
    // are left as they were when a vector is refused.
    cuda_check(cudaMemsetAsync(bad, 0, sizeof(unsigned), 0), "pool check");
    cuda_check(qm::launch_count_non_unit(stage_dirs, n, bad, 0), "pool check");
    cuda_check(qm::launch_count_non_unit(stage_pert, n, bad, 0), "pool check");
    unsigned h_bad = 0;
    cuda_check(cudaMemcpy(&h_bad, bad, sizeof(unsigned), cudaMemcpyDeviceToHost), "pool check");
    if (h_bad) invalid("sample-pool vectors must be unit vectors (squared length in [0.25, 4])");
    cuda_check(qm::launch_xyz_to_float4(stage_dirs, s->d_samples.as<float4>(), n, 0), "pool convert");
    cuda_check(qm::launch_xyz_to_float4(stage_pert, s->d_perturb.as<float4>(), n, 0), "pool convert");
    cuda_check(cudaDeviceSynchronize(), "pool convert");
    rotate_pool(s, true);
  });
}

int qmcrt_generate_sample_pool(qmcrt_scene* s, unsigned seed, int sunshape, float half_angle) {
  return guarded([&] {
    checked(s);
    if (sunshape == qm::kSunshapePillbox && !(half_angle > 0.0f && half_angle < 1.0f))
      invalid("pillbox half-angle must be in (0, 1) radians");
    DeviceGuard guard(s->device);
    generate_pool(s, seed, sunshape, half_angle);
  });
}

int qmcrt_get_sample_pool(qmcrt_scene* s, float* dirs, float* perturb) {
  return guarded([&] {
    checked(s);
    DeviceGuard guard(s->device);
    std::vector<float4> tmp(s->pool_size);
    if (dirs) {
      cuda_check(cudaMemcpy(tmp.data(), s->d_samples.p, tmp.size() * sizeof(float4), cudaMemcpyDeviceToHost), "readback");
      for (size_t i = 0; i < tmp.size(); ++i) dirs[3 * i] = tmp[i].x, dirs[3 * i + 1] = tmp[i].y, dirs[3 * i + 2] = tmp[i].z;
    }
    if (perturb) {
      cuda_check(cudaMemcpy(tmp.data(), s->d_perturb.p, tmp.size() * sizeof(float4), cudaMemcpyDeviceToHost), "readback");
      for (size_t i = 0; i < tmp.size(); ++i)
        perturb[3 * i] = tmp[i].x, perturb[3 * i + 1] = tmp[i].y, perturb[3 * i + 2] = tmp[i].z;
    }
  });
}

int qmcrt_set_facet_offsets(qmcrt_scene* s, int id, const int* offsets, int n) {
  return guarded([&] {
    checked(s);
    check_heliostat(s, id);
    const int nf = s->model.heliostats[id].num_facets;
    if (!offsets || (n != nf && n != nf + 1)) invalid("offsets must hold num_facets or num_facets + 1 entries");
    std::vector<int> v(offsets, offsets + n);
    if (n == nf) v.push_back(nf > 0 ? v[0] : 0);
    for (int x : v)
      if (x < 0 || x >= s->pool_size) invalid("facet offsets must lie in [0, pool_size)");
    DeviceGuard guard(s->device);
    cuda_check(cudaMemcpy(s->d_offsets.as<int>() + s->offset_base[id], v.data(), v.size() * sizeof(int),
                          cudaMemcpyHostToDevice),
               "offsets upload");
  });
}

int qmcrt_get_facet_offsets(qmcrt_scene* s, int id, int* offsets, int n) {
  return guarded([&] {
    checked(s);
    check_heliostat(s, id);
    const int nf = s->model.heliostats[id].num_facets;
    if (!offsets || n < 0 || n > nf + 1) invalid("offsets buffer size out of range");
    DeviceGuard guard(s->device);
    cuda_check(cudaMemcpy(offsets, s->d_offsets.as<int>() + s->offset_base[id], (size_t)n * sizeof(int),
                          cudaMemcpyDeviceToHost),
               "offsets readback");
  });
}

int qmcrt_generate_facet_offsets(qmcrt_scene* s, unsigned seed) {
  return guarded([&] {
    checked(s);
    DeviceGuard guard(s->device);
    generate_offsets(s, seed);
  });
}

int qmcrt_set_math_mode(qmcrt_scene* s, int exact) {
  return guarded([&] {
    if (exact < 0 || exact > 4)
      invalid("math mode must be 0 (production), 1 (exact), 2 (production, 64 registers), 3 (approximate math) or "
              "4 (production, approximate receiver arithmetic)");
    checked(s)->exact = exact;
  });
}

int qmcrt_set_light_range(qmcrt_scene* s, int begin, int end) {
  return guarded([&] {
    checked(s);
    if (begin < 0 || end < begin || end > s->model.config.num_per_sunshape_group)
      invalid("light range must satisfy 0 <= begin <= end <= num_per_sunshape_group");
    s->light_begin = begin;
    s->light_end = end;
  });
}

int qmcrt_trace_heliostat(qmcrt_scene* s, int id, void* stream) {
  return guarded([&] { trace_ids(checked(s), &id, 1, static_cast<cudaStream_t>(stream)); });
}

int qmcrt_trace_heliostats(qmcrt_scene* s, const int* ids, int n, void* stream) {
  return guarded([&] { trace_ids(checked(s), ids, n, static_cast<cudaStream_t>(stream)); });
}

int qmcrt_launch_shapes(int* threads, int* chunk_iters, int* persistent, int* count) {
  return guarded([&] {
    if (count) *count = kNumShapes;
    for (int k = 0; k < kNumShapes; ++k) {
      if (threads) threads[k] = kShapes[k].threads;
      if (chunk_iters) chunk_iters[k] = kShapes[k].chunk_iters;
      if (persistent) persistent[k] = kShapes[k].persistent;
    }
  });
}

int qmcrt_set_launch_shape(qmcrt_scene* s, int shape) {
  return guarded([&] {
    checked(s);
    if (shape < 0 || shape >= kNumShapes) invalid("launch shape out of range");
    s->shape = shape;
  });
}

int qmcrt_autotune(qmcrt_scene* s, const int* ids, int n, void* stream, int* best, float* ms_per_shape) {
  return guarded([&] {
    checked(s);
    if (s->exact != 0) throw ApiError(QMCRT_ERR_STATE, "the launch shapes belong to the production build (math mode 0)");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    DeviceGuard guard(s->device);
    cudaEvent_t e0, e1;
    cuda_check(cudaEventCreate(&e0), "cudaEventCreate");
    cuda_check(cudaEventCreate(&e1), "cudaEventCreate");
    float best_ms = 1e30f;
    int pick = 0;
    for (int k = 0; k < kNumShapes; ++k) {
      s->shape = k;
      trace_ids(s, ids, n, st);  // warm-up (and the task upload for this chunk size)
      cuda_check(cudaEventRecord(e0, st), "cudaEventRecord");
      trace_ids(s, ids, n, st);
      cuda_check(cudaEventRecord(e1, st), "cudaEventRecord");
      cuda_check(cudaEventSynchronize(e1), "autotune");
      float t = 0.f;
      cudaEventElapsedTime(&t, e0, e1);
      if (ms_per_shape) ms_per_shape[k] = t;
      if (t < best_ms) {
        best_ms = t;
        pick = k;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    s->shape = pick;
    for (auto& img : s->images) cuda_check(cudaMemsetAsync(img->p, 0, img->bytes, st), "image clear");
    cuda_check(cudaStreamSynchronize(st), "autotune");
    cuda_check(cudaMemset(s->d_power.p, 0, s->d_power.bytes), "clear");
    if (best) *best = pick;
  });
}

int qmcrt_debug_hit_bits(qmcrt_scene* s, const int* ids, int n, unsigned* device_bits, long long capacity,
                         long long* words, void* stream) {
  return guarded([&] {
    checked(s);
    if (capacity < 0) invalid("capacity must not be negative");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const long long need = trace_ids(s, ids, n, st, 3, nullptr) * qm::kChunkIters;
    if (words) *words = need;
    if (!device_bits) return;
    if (capacity < need) invalid("the bit buffer holds fewer words than the launch needs");
    DeviceGuard guard(s->device);
    if (need > 0) cuda_check(cudaMemsetAsync(device_bits, 0, (size_t)need * sizeof(uint32_t), st), "clear bits");
    trace_ids(s, ids, n, st, 3, reinterpret_cast<uint32_t*>(device_bits));
  });
}

int qmcrt_receiver_image(qmcrt_scene* s, int id, float* out, int* width, int* height) {
  return guarded([&] {
    checked(s);
    if (id < 0 || id >= (int)s->model.receivers.size()) invalid("receiver index out of range");
    const auto& r = s->model.receivers[id];
    if (width) *width = r.resolution.x;
    if (height) *height = r.resolution.y;
    if (out) {
      DeviceGuard guard(s->device);
      cuda_check(cudaDeviceSynchronize(), "synchronise");
      cuda_check(cudaMemcpy(out, s->images[id]->p, (size_t)r.resolution.x * r.resolution.y * sizeof(float),
                            cudaMemcpyDeviceToHost),
                 "image readback");
    }
  });
}

int qmcrt_receiver_device_image(qmcrt_scene* s, int id, float** dptr, int* width, int* height) {
  return guarded([&] {
    checked(s);
    if (id < 0 || id >= (int)s->model.receivers.size()) invalid("receiver index out of range");
    const auto& r = s->model.receivers[id];
    if (dptr) *dptr = s->images[id]->as<float>();
    if (width) *width = r.resolution.x;
    if (height) *height = r.resolution.y;
  });
}

int qmcrt_receiver_clear(qmcrt_scene* s, int id, void* stream) {
  return guarded([&] {
    checked(s);
    if (id < 0 || id >= (int)s->model.receivers.size()) invalid("receiver index out of range");
    DeviceGuard guard(s->device);
    cuda_check(cudaMemsetAsync(s->images[id]->p, 0, s->images[id]->bytes, static_cast<cudaStream_t>(stream)),
               "image clear");
  });
}

int qmcrt_power_fp64(qmcrt_scene* s, double* per, double* total) {
  return guarded([&] {
    checked(s);
    DeviceGuard guard(s->device);
    std::vector<double> v(s->model.heliostats.size());
    cuda_check(cudaDeviceSynchronize(), "synchronise");
    if (!v.empty())
      cuda_check(cudaMemcpy(v.data(), s->d_power.p, v.size() * sizeof(double), cudaMemcpyDeviceToHost), "readback");
    if (per) std::copy(v.begin(), v.end(), per);
    if (total) {
      // Neumaier-compensated sum of the per-heliostat totals.
      double sum = 0.0, comp = 0.0;
      for (double x : v) {
        double t = sum + x;
        comp += (std::fabs(sum) >= std::fabs(x)) ? (sum - t) + x : (x - t) + sum;
        sum = t;
      }
      *total = sum + comp;
    }
  });
}

int qmcrt_power_clear(qmcrt_scene* s) {
  return guarded([&] {
    checked(s);
    DeviceGuard guard(s->device);
    cuda_check(cudaDeviceSynchronize(), "synchronise");
    cuda_check(cudaMemset(s->d_power.p, 0, s->d_power.bytes), "clear");
    cuda_check(cudaMemset(s->d_diag.p, 0, s->d_diag.bytes), "clear");
  });
}

int qmcrt_diagnostics(qmcrt_scene* s, unsigned long long* out4) {
  return guarded([&] {
    checked(s);
    if (!out4) invalid("output is NULL");
    DeviceGuard guard(s->device);
    cuda_check(cudaDeviceSynchronize(), "synchronise");
    cuda_check(cudaMemcpy(out4, s->d_diag.p, qm::kDiagSlots * sizeof(unsigned long long), cudaMemcpyDeviceToHost),
               "readback");
  });
}

int qmcrt_debug_shadow_free(qmcrt_scene* s, int* flags) {
  return guarded([&] {
    checked(s);
    if (!flags) invalid("output is NULL");
    for (size_t i = 0; i < s->templates.size(); ++i) flags[i] = s->templates[i].shadow_free;
  });
}

int qmcrt_grid_build_device(qmcrt_scene* s, int grid, float* ms) {
  return guarded([&] {
    checked(s);
    if (grid < 0 || grid >= (int)s->model.grids.size()) invalid("grid index out of range");
    const qm::GridModel& g = s->model.grids[grid];
    GridBufs& gb = *s->grid_bufs[grid];
    DeviceGuard guard(s->device);
    // Inputs: each heliostat's position and half size length (as the host
    // grid builder forms them) and its sub-heliostat range.
    std::vector<float4> pr(std::max(g.num_heliostats, 1));
    std::vector<int2> subs(std::max(g.num_heliostats, 1));
    for (int i = 0; i < g.num_heliostats; ++i) {
      const qm::HeliostatModel& h = s->model.heliostats[g.start_heliostat + i];
      const float radius = qm::length(h.size) / 2;
      pr[i] = make_float4(h.pos.x, h.pos.y, h.pos.z, radius);
      subs[i] = make_int2(h.sub_begin, h.num_sub);
    }
    const long long ncell = (long long)g.cells.x * g.cells.y * g.cells.z;
    DBuf d_pr, d_subs, d_counts, d_ranges, d_total, d_entries;
    upload(d_pr, pr);
    upload(d_subs, subs);
    d_counts.alloc((size_t)ncell * sizeof(int));
    d_ranges.alloc((size_t)ncell * sizeof(int2));
    d_total.alloc(sizeof(int));
    qm::GridBuildParams p{};
    p.pos = g.pos;
    p.interval = g.interval;
    p.cells = g.cells;
    p.num_heliostats = g.num_heliostats;
    p.pos_radius = d_pr.as<float4>();
    p.subs = d_subs.as<int2>();
    p.counts = d_counts.as<int>();
    p.ranges = d_ranges.as<int2>();
    p.total = d_total.as<int>();
    cudaEvent_t e0, e1, e2;
    cuda_check(cudaEventCreate(&e0), "cudaEventCreate");
    cuda_check(cudaEventCreate(&e1), "cudaEventCreate");
    cuda_check(cudaEventCreate(&e2), "cudaEventCreate");
    cuda_check(cudaEventRecord(e0, 0), "cudaEventRecord");
    cuda_check(qm::launch_grid_count(p, 0), "grid count");
    cuda_check(cudaEventRecord(e1, 0), "cudaEventRecord");
    int total = 0;
    cuda_check(cudaMemcpy(&total, d_total.p, sizeof(int), cudaMemcpyDeviceToHost), "grid total");
    float t_count = 0.f, t_fill = 0.f;
    cuda_check(cudaEventElapsedTime(&t_count, e0, e1), "cudaEventElapsedTime");
    const size_t want = gb.entries.bytes / sizeof(int4);
    if ((size_t)total != want) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      cudaEventDestroy(e2);
      throw ApiError(QMCRT_ERR_INVALID, "device grid build found " + std::to_string(total) + " entries, the scene holds " +
                                            std::to_string(want));
    }
    d_entries.alloc(std::max<size_t>(total, 1) * sizeof(int4));
    p.entries = d_entries.as<int4>();
    cuda_check(cudaEventRecord(e1, 0), "cudaEventRecord");
    cuda_check(qm::launch_grid_fill(p, 0), "grid fill");
    cuda_check(cudaEventRecord(e2, 0), "cudaEventRecord");
    cuda_check(cudaEventSynchronize(e2), "grid build");
    cuda_check(cudaEventElapsedTime(&t_fill, e1, e2), "cudaEventElapsedTime");
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(e2);
    // The scene's lists are replaced in place (same sizes), so batches that
    // share them keep valid pointers.
    cuda_check(cudaDeviceSynchronize(), "synchronise");
    cuda_check(cudaMemcpy(gb.ranges.p, d_ranges.p, (size_t)ncell * sizeof(int2), cudaMemcpyDeviceToDevice),
               "grid ranges");
    if (total > 0)
      cuda_check(cudaMemcpy(gb.entries.p, d_entries.p, (size_t)total * sizeof(int4), cudaMemcpyDeviceToDevice),
                 "grid entries");
    if (ms) *ms = t_count + t_fill;
  });
}

int qmcrt_debug_grid_cells(qmcrt_scene* s, int grid, int* ranges, int* entries, long long* num_entries) {
  return guarded([&] {
    checked(s);
    if (grid < 0 || grid >= (int)s->model.grids.size()) invalid("grid index out of range");
    const qm::GridModel& g = s->model.grids[grid];
    GridBufs& gb = *s->grid_bufs[grid];
    const long long ncell = (long long)g.cells.x * g.cells.y * g.cells.z;
    const long long n = (long long)(gb.entries.bytes / sizeof(int4));
    if (num_entries) *num_entries = n;
    DeviceGuard guard(s->device);
    if (ranges)
      cuda_check(cudaMemcpy(ranges, gb.ranges.p, (size_t)ncell * sizeof(int2), cudaMemcpyDeviceToHost), "readback");
    if (entries && n > 0)
      cuda_check(cudaMemcpy(entries, gb.entries.p, (size_t)n * sizeof(int4), cudaMemcpyDeviceToHost), "readback");
  });
}

int qmcrt_debug_block_free(qmcrt_scene* s, int grid, int* flags) {
  return guarded([&] {
    checked(s);
    if (!flags) invalid("output is NULL");
    if (grid < 0 || grid >= (int)s->model.grids.size()) invalid("grid index out of range");
    const int n = s->model.grids[grid].num_subheliostats;
    DeviceGuard guard(s->device);
    cuda_check(cudaMemcpy(flags, s->grid_bufs[grid]->sub_free.p, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost),
               "flag readback");
  });
}

int qmcrt_debug_hit_records(qmcrt_scene* s, int id, int fb, int fe, int lb, int le, int* codes) {
  return guarded([&] {
    checked(s);
    check_heliostat(s, id);
    const int nf = s->model.heliostats[id].num_facets;
    if (fb < 0 || fe < fb || fe > nf) invalid("facet range out of bounds");
    if (lb < 0 || le < lb || le > s->model.config.num_per_sunshape_group) invalid("light range out of bounds");
    if (!codes) invalid("output is NULL");
    if ((long long)fe * (le - lb) > kMaxTaskRays) invalid("facet_end x lights must stay below 2^31 - 2^16");
    const size_t count = (size_t)(fe - fb) * (le - lb);
    if (count == 0) return;
    DeviceGuard guard(s->device);
    // Scratch receivers, power and counters so the scene's state is untouched.
    std::vector<DevReceiver> recv = s->receivers;
    size_t maxpix = 1;
    for (auto& r : recv) maxpix = std::max(maxpix, (size_t)r.resolution.x * r.resolution.y);
    DBuf img, dr, rec, pw, dg, task, prefix;
    img.alloc(maxpix * sizeof(float));
    for (auto& r : recv) r.image = img.as<float>();
    upload(dr, recv);
    rec.alloc(count * sizeof(int32_t));
    pw.alloc(s->model.heliostats.size() * sizeof(double) + 8);
    dg.alloc(qm::kDiagSlots * sizeof(unsigned long long));
    std::vector<DevTask> one{s->templates[id]};
    upload(task, one);
    qm::TraceParams p = base_params(s);
    p.receivers = dr.as<DevReceiver>();
    p.tasks = task.as<DevTask>();
    p.num_tasks = 1;
    p.power = pw.as<double>();
    p.diag = dg.as<unsigned long long>();
    p.light_begin = lb;
    p.light_end = le;
    p.records = rec.as<int32_t>();
    p.record_task = 0;
    p.record_facet_begin = fb;
    p.record_facet_end = fe;
    cuda_check(run_trace(s, p, 1, 0), "record kernel");
    cuda_check(cudaMemcpy(codes, rec.p, count * sizeof(int32_t), cudaMemcpyDeviceToHost), "readback");
  });
}

int qmcrt_smooth(float* d_img, int width, int height, int radius, float ratio, void* stream) {
  return guarded([&] {
    if (!d_img) invalid("image is NULL");
    if (width <= 0 || height <= 0) invalid("image size must be positive");
    if (radius < 0 || radius > 64) invalid("radius must be in [0, 64]");
    if (!(ratio >= 0.0f && ratio < 0.5f)) invalid("trim ratio must be in [0, 0.5)");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t bytes = (size_t)width * height * sizeof(float);
    void* copy = nullptr;
    alloc_gate("cudaMallocAsync");
    cuda_check(cudaMallocAsync(&copy, bytes, st), "cudaMallocAsync");
    cudaError_t e = cudaMemcpyAsync(copy, d_img, bytes, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = qm::launch_trimmed_mean(static_cast<float*>(copy), d_img, width, height, radius, ratio, st);
    cudaFreeAsync(copy, st);
    cuda_check(e, "trimmed mean");
  });
}

int qmcrt_load_tasks(const qmcrt_scene* s, const char* path, int* hs, int* nh, int capacity, int* rs, int* nr,
                     int* status) {
  return guarded([&] {
    if (!s || !path) invalid("scene or path is NULL");
    std::vector<int> h, r;
    std::string err;
    int st = qm::read_task_file(path, s->model, h, r, err);
    if (st < 0) throw ApiError(QMCRT_ERR_IO, err);
    if ((int)h.size() > capacity || (int)r.size() > capacity) invalid("task buffers are too small");
    if (hs) std::copy(h.begin(), h.end(), hs);
    if (rs) std::copy(r.begin(), r.end(), rs);
    if (nh) *nh = (int)h.size();
    if (nr) *nr = (int)r.size();
    if (status) *status = st;
  });
}

int qmcrt_save_text(const char* path, int height, int width, const float* data, int precision, float* max_value) {
  return guarded([&] {
    if (!path || !data || height < 0 || width < 0 || precision < 0 || precision > 30) invalid("bad arguments");
    std::string err;
    bool ok = false;
    float m = qm::save_text_image(path, height, width, data, precision, err, &ok);
    if (!ok) throw ApiError(QMCRT_ERR_IO, err);
    if (max_value) *max_value = m;
  });
}

}  // extern "C"
