// CPU ORACLE - test infrastructure only.
//
// C entry points over the reference's own host code, compiled from the
// reference tree by oracle/build_ref.py into oracle/_ref/libref_host.so and
// linked against host_cudart.cpp (no GPU needed).  Tests use it to pin the
// oracle restatement (qmcrt_oracle.cpp) to the reference's behaviour, and
// bench.py uses its per-ray loop as the CPU baseline ("reference" kind).
//
// What runs here is the reference's code: SceneConfiguration, SceneLoader,
// SceneProcessor::set_grid_receiver_heliostat_content, RectangleGrid,
// receivers, heliostats (CSetNormalAndRotate, CGetSubHeliostatVertexes),
// rectGridDDA::collision, GIntersect, calEnergy, samplelights::parameters_generate,
// max_less_index, the smoother's heap classes, TaskLoader, ImageSaver.
// Restated here (the reference has them only as __global__ kernel bodies or
// device-only functions): the per-ray loop of map_raytracing with
// receiver_drawing's pixel arithmetic, the focus-flat micro-facet kernels,
// linear_interpolation's body and trimmed_mean's loop.  They call the
// reference's inline helpers for every arithmetic step.
#include <fcntl.h>
#include <omp.h>
#include <unistd.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <iostream>
#include <memory>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <unordered_set>
#include <vector>

#include <cuda_runtime.h>

#define private public
#define protected public
#include "CylinderReceiver.cuh"
#include "FocusFlatRectangleHelio.cuh"
#include "Grid/rectGridDDA.cuh"
#include "ImageSaver/ImageSaver.h"
#include "RayTracingArgumentStruct.h"
#include "RectangleGrid.cuh"
#include "RectangleHelio.cuh"
#include "RectangleReceiver.cuh"
#include "Receiver/receiverIntersectionUtil.cuh"
#include "SceneConfiguration.h"
#include "SceneLoader.h"
#include "SceneProcessor.h"
#include "Smoother/heap.cuh"
#include "SolarScene.h"
#include "TaskLoader.h"
#include "global_function.cuh"
#undef private
#undef protected

// Reference host functions defined in .cu files without a header declaration.
void host_map_microhelio_center_and_normal(int myId, float3* d_microhelio_centers, float3* d_microhelio_normals,
                                           float3 normal, float3 helio_size, const int2 row_col,
                                           const int2 sub_row_col, const float pixel_length, const float2 gap,
                                           const float3 world_pos, const size_t map_size);
namespace samplelights {
float integration_larger_than_465_intensity(float theta, float k, float gamma);
float2* parameters_generate(float* h_k, int num_group, float k, float gamma, float upper_lm);
__host__ __device__ int max_less_index(float2* d_cdf, float value, size_t n);
}  // namespace samplelights

// Heliostat type is not stored by the reference; recover it from the class.
int Heliostat_type(Heliostat* h) { return dynamic_cast<FocusFlatRectangleHelio*>(h) ? 1 : 0; }

namespace {

// Silences the reference's printf/cout chatter (stdout) for a scope.
struct Quiet {
  int saved = -1;
  Quiet() {
    std::fflush(stdout);
    std::cout.flush();
    saved = dup(1);
    int devnull = open("/dev/null", O_WRONLY);
    if (devnull >= 0) {
      dup2(devnull, 1);
      close(devnull);
    }
  }
  ~Quiet() {
    std::fflush(stdout);
    std::cout.flush();
    if (saved >= 0) {
      dup2(saved, 1);
      close(saved);
    }
  }
};

std::string g_err;
TaskLoader g_tasks;

// Empties the SolarScene singleton.  SolarScene::clear() is not called: it
// falls off the end of a bool function (Scene/SolarScene.cpp:31-46), which is
// undefined behaviour and crashes when compiled with optimisation.  The
// previous scene's objects are leaked (test processes are short-lived).
void clear_scene() {
  SolarScene* s = SolarScene::GetInstance();
  s->receivers.clear();
  s->grids.clear();
  s->heliostats.clear();
}

void reset_singletons() {
  clear_scene();
  delete SceneConfiguration::sceneConfigurationInstance;
  SceneConfiguration::sceneConfigurationInstance = nullptr;
}

int sub_begin_of(int hid) {
  // QuasiMonteCarloRayTracer::generateHeliostatArgument (QuasiMonteCarloRayTracer.cpp:148-158).
  SolarScene* s = SolarScene::GetInstance();
  Grid* g = s->getGrids()[s->getHeliostats()[hid]->getBelongingGridId()];
  int id = 0;
  for (int i = 0; i < g->getNumberOfHeliostats(); ++i) {
    int real = i + g->getStartHeliostatIndex();
    if (real == hid) break;
    id += s->getHeliostats()[real]->getSubHelioSize();
  }
  return id;
}

// Micro-facet count and lattice (RectangleHelio.cu:84-104 / FocusFlatRectangleHelio.cu:68-82).
void lattice(Heliostat* h, int2& sub_row_col, float2& len, int& n) {
  int2 rc = h->getRowAndColumn();
  float3 size = h->getSize();
  float2 gap = h->getGap();
  len.x = (size.z - gap.y * (rc.x - 1)) / float(rc.x);
  len.y = (size.x - gap.x * (rc.y - 1)) / float(rc.y);
  sub_row_col.x = int(len.x / h->getPixelLength());
  sub_row_col.y = int(len.y / h->getPixelLength());
  n = rc.x * rc.y * sub_row_col.x * sub_row_col.y;
}

// Focus-flat micro-facet f (the focus-flat branch; flat heliostats use the
// reference's host_map_microhelio_center_and_normal directly).
void facet(Heliostat* h, int f, const int2& sub_row_col, const float2& len, int n, float3& o, float3& nn) {
  (void)n;
  // focusFlatRectangle_heliostat kernels (FocusFlatRectangleHelio.cu:12-64), body by body.
  auto* ff = static_cast<FocusFlatRectangleHelio*>(h);
  int2 rc = h->getRowAndColumn();
  int row = f / (rc.y * sub_row_col.y);
  int col = f % (rc.y * sub_row_col.y);
  int block = global_func::unroll_index(make_int2(row / sub_row_col.x, col / sub_row_col.y), rc);
  float3 ln = ff->d_local_normals[block];
  float3 lc = ff->d_local_centers[block];
  row %= sub_row_col.x;
  col %= sub_row_col.y;
  float3 subhelio_size = make_float3(len.y, h->getSize().y, len.x);
  float3 lp = make_float3((col + 0.5f) * h->getPixelLength() - subhelio_size.x / 2, 0.0f,
                          (row + 0.5f) * h->getPixelLength() - subhelio_size.z / 2);
  lp = focusFlatRectangle_heliostat::focusFlatRectangleHeliostatLocal2WorldRotate(lp, ln);
  lp = global_func::translate(lp, lc);
  nn = focusFlatRectangle_heliostat::focusFlatRectangleHeliostatLocal2WorldRotate(ln, h->getNormal());
  o = focusFlatRectangle_heliostat::focusFlatRectangleHeliostatLocal2WorldRotate(lp, h->getNormal());
  o = global_func::translate(o, h->getPosition());
}

}  // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

// SceneConfiguration::loadConfiguration on a fresh singleton: fields set, or -1 on throw.
int ref_load_config(const char* path) {
  Quiet quiet;
  delete SceneConfiguration::sceneConfigurationInstance;
  SceneConfiguration::sceneConfigurationInstance = nullptr;
  try {
    std::streambuf* old = std::cout.rdbuf(nullptr);
    int n = SceneConfiguration::getInstance()->loadConfiguration(path);
    std::cout.rdbuf(old);
    return n;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

// SceneLoader::SceneFileRead on a cleared scene: 1 / 0.
int ref_read_scene(const char* path) {
  Quiet quiet;
  reset_singletons();
  SceneLoader loader;
  std::streambuf* old = std::cerr.rdbuf(nullptr);
  bool ok = loader.SceneFileRead(SolarScene::GetInstance(), path);
  std::cerr.rdbuf(old);
  return ok ? 1 : 0;
}

// Configuration + scene + the geometry half of processScene. counts3 = receivers, grids, heliostats.
int ref_load(const char* scene_path, const char* config_path, int* counts3) {
  Quiet quiet;
  if (ref_load_config(config_path) < 0) return -1;
  SolarScene* s = SolarScene::GetInstance();
  clear_scene();
  SceneLoader loader;
  std::streambuf* oldc = std::cout.rdbuf(nullptr);
  std::streambuf* olde = std::cerr.rdbuf(nullptr);
  bool ok = loader.SceneFileRead(s, scene_path);
  if (ok) {
    SceneProcessor proc(SceneConfiguration::getInstance());
    proc.set_grid_receiver_heliostat_content(s->getGrids(), s->getReceivers(), s->getHeliostats());
    // Sub-heliostat tables for every grid (fills focus-flat local frames).
    for (Grid* g : s->getGrids()) {
      std::vector<float3> v;
      for (int i = g->getStartHeliostatIndex(); i < g->getStartHeliostatIndex() + g->getNumberOfHeliostats(); ++i)
        s->getHeliostats()[i]->CGetSubHeliostatVertexes(v);
    }
  }
  std::cout.rdbuf(oldc);
  std::cerr.rdbuf(olde);
  if (!ok) return -2;
  counts3[0] = (int)s->getReceivers().size();
  counts3[1] = (int)s->getGrids().size();
  counts3[2] = (int)s->getHeliostats().size();
  return 0;
}

void ref_receiver(int i, int* ints3, float* vals19) {
  Receiver* r = SolarScene::GetInstance()->getReceivers()[i];
  ints3[0] = r->getType();
  ints3[1] = r->getResolution().x;
  ints3[2] = r->getResolution().y;
  vals19[0] = r->getPixelLength();
  std::fill(vals19 + 1, vals19 + 19, 0.0f);
  if (r->getType() == 0) {
    auto* rr = static_cast<RectangleReceiver*>(r);
    for (int k = 0; k < 4; ++k) {
      float3 v = rr->getRectangleVertex(k);
      vals19[1 + 3 * k] = v.x, vals19[2 + 3 * k] = v.y, vals19[3 + 3 * k] = v.z;
    }
    float3 f = rr->focus_center_;
    vals19[16] = f.x, vals19[17] = f.y, vals19[18] = f.z;
  }
  float3 n = r->getNormal();
  vals19[13] = n.x, vals19[14] = n.y, vals19[15] = n.z;
}

// type, grid, n_facets, n_sub, sub_begin | normal3, focus_length
void ref_heliostat(int i, int* ints5, float* vals4) {
  Heliostat* h = SolarScene::GetInstance()->getHeliostats()[i];
  int2 src;
  float2 len;
  int n;
  lattice(h, src, len, n);
  ints5[0] = Heliostat_type(h);
  ints5[1] = h->getBelongingGridId();
  ints5[2] = n;
  ints5[3] = h->getSubHelioSize();
  ints5[4] = sub_begin_of(i);
  float3 nn = h->getNormal();
  vals4[0] = nn.x, vals4[1] = nn.y, vals4[2] = nn.z;
  vals4[3] = ints5[0] == 1 ? static_cast<FocusFlatRectangleHelio*>(h)->getFocusLength() : -1.0f;
}

// cells3, nnz, n_sub_heliostats
void ref_grid(int i, int* ints5) {
  Quiet quiet;
  auto* g = static_cast<RectangleGrid*>(SolarScene::GetInstance()->getGrids()[i]);
  int3 c = g->getSubGridNumber();
  ints5[0] = c.x, ints5[1] = c.y, ints5[2] = c.z;
  ints5[3] = (int)g->getNumberOfGridHeliostatMatch();
  std::vector<float3> v;
  for (int k = g->getStartHeliostatIndex(); k < g->getStartHeliostatIndex() + g->getNumberOfHeliostats(); ++k)
    SolarScene::GetInstance()->getHeliostats()[k]->CGetSubHeliostatVertexes(v);
  ints5[4] = (int)v.size() / 3;
}

void ref_grid_csr(int i, int* index, int* match) {
  auto* g = static_cast<RectangleGrid*>(SolarScene::GetInstance()->getGrids()[i]);
  int3 c = g->getSubGridNumber();
  std::memcpy(index, g->getDeviceGridHeliostatIndex(), sizeof(int) * (size_t)(c.x * c.y * c.z + 1));
  std::memcpy(match, g->getDeviceGridHeliostatMatch(), sizeof(int) * g->getNumberOfGridHeliostatMatch());
}

// QuasiMonteCarloRayTracer::setFlatRectangleHeliostatVertexs's table.
void ref_grid_vertices(int i, float* xyz) {
  Quiet quiet;
  SolarScene* s = SolarScene::GetInstance();
  Grid* g = s->getGrids()[i];
  std::vector<float3> v;
  for (int k = g->getStartHeliostatIndex(); k < g->getStartHeliostatIndex() + g->getNumberOfHeliostats(); ++k)
    s->getHeliostats()[k]->CGetSubHeliostatVertexes(v);
  for (size_t k = 0; k < v.size(); ++k) xyz[3 * k] = v[k].x, xyz[3 * k + 1] = v[k].y, xyz[3 * k + 2] = v[k].z;
}

void all_facets(Heliostat* h, std::vector<float3>& o, std::vector<float3>& nn) {
  int2 src;
  float2 len;
  int n;
  lattice(h, src, len, n);
  o.assign(n, make_float3(0, 0, 0));
  nn.assign(n, make_float3(0, 0, 0));
#pragma omp parallel for schedule(static)
  for (int f = 0; f < n; ++f) {
    if (Heliostat_type(h) == 0) {
      host_map_microhelio_center_and_normal(f, o.data(), nn.data(), h->getNormal(), h->getSize(),
                                            h->getRowAndColumn(), src, h->getPixelLength(), h->getGap(),
                                            h->getPosition(), (size_t)n);
    } else {
      facet(h, f, src, len, n, o[f], nn[f]);
    }
  }
}

void ref_facets(int i, float* origins, float* normals) {
  Heliostat* h = SolarScene::GetInstance()->getHeliostats()[i];
  std::vector<float3> o, nn;
  all_facets(h, o, nn);
  const int n = (int)o.size();
  for (int f = 0; f < n; ++f) {
    origins[3 * f] = o[f].x, origins[3 * f + 1] = o[f].y, origins[3 * f + 2] = o[f].z;
    normals[3 * f] = nn[f].x, normals[3 * f + 1] = nn[f].y, normals[3 * f + 2] = nn[f].z;
  }
}

// rectGridDDA::collision for one ray, with heliostat `hid`'s own sub-heliostats skipped.
int ref_collision(int hid, const float* o, const float* d) {
  Quiet quiet;
  SolarScene* s = SolarScene::GetInstance();
  Heliostat* h = s->getHeliostats()[hid];
  auto* g = static_cast<RectangleGrid*>(s->getGrids()[h->getBelongingGridId()]);
  std::vector<float3> v;
  for (int k = g->getStartHeliostatIndex(); k < g->getStartHeliostatIndex() + g->getNumberOfHeliostats(); ++k)
    s->getHeliostats()[k]->CGetSubHeliostatVertexes(v);
  HeliostatArgument arg(nullptr, nullptr, nullptr, 0, sub_begin_of(hid), h->getSubHelioSize());
  bool hit = rectGridDDA::collision(make_float3(o[0], o[1], o[2]), make_float3(d[0], d[1], d[2]), *g, v.data(), arg);
  return hit ? 1 : 0;
}

// Receiver GIntersect for one ray: 1 on a hit, tuv filled.
int ref_receiver_hit(int r, const float* o, const float* d, float* tuv) {
  Receiver* rc = SolarScene::GetInstance()->getReceivers()[r];
  float t = 0, u = 0, v = 0;
  bool hit;
  float3 oo = make_float3(o[0], o[1], o[2]), dd = make_float3(d[0], d[1], d[2]);
  if (rc->getType() == 0) hit = static_cast<RectangleReceiver*>(rc)->GIntersect(oo, dd, t, u, v);
  else hit = static_cast<CylinderReceiver*>(rc)->GIntersect(oo, dd, t, u, v);
  tuv[0] = t, tuv[1] = u, tuv[2] = v;
  return hit ? 1 : 0;
}

struct RefTraceArgs {
  const int* ids;
  int n_ids;
  const float* pool_dirs;
  const float* pool_pert;
  int pool_size;
  const int* offsets;
  const long long* offset_base;
  int light_begin, light_end;
  int facet_stride, facet_phase;
  double* images;
  const long long* image_base;
  double* power;
  long long* counters;  // rays, shadowed, blocked, missed, hit, clamped
  int rec_id, rec_facet_begin, rec_facet_end;
  int* records;
  int threads;
};

// The per-ray body of map_raytracing (RectangleReceiverRectangleGridRayTracing.cu:6-41,
// CylinderReceiverRectangleGridRayTracing.cu:6-40) and receiver_drawing
// (rectangleReceiverIntersection.cu:8-26, cylinderReceiverIntersection.cu:4-21)
// as a host loop: OpenMP over facets, per-thread double images.  Pixel
// indexes that would fall outside the image (u or v == 1) are clamped and counted.
void ref_trace(const RefTraceArgs* a) {
  Quiet quiet;
  SolarScene* s = SolarScene::GetInstance();
  SceneConfiguration* cfg = SceneConfiguration::getInstance();
  float3 sun_dir = cfg->getSun_dir();
  const int L = cfg->getNum_sunshape_lights_per_group();
  const int P = a->pool_size;
  const long long total_pix = a->images ? a->image_base[s->getReceivers().size()] : 0;
  long long totals[6] = {0};
  if (a->threads > 0) omp_set_num_threads(a->threads);
  // Sub-heliostat vertex table of each grid (setFlatRectangleHeliostatVertexs), built once.
  std::vector<std::vector<float3>> grid_verts(s->getGrids().size());
  for (size_t gi = 0; gi < s->getGrids().size(); ++gi) {
    Grid* g = s->getGrids()[gi];
    for (int k = g->getStartHeliostatIndex(); k < g->getStartHeliostatIndex() + g->getNumberOfHeliostats(); ++k)
      s->getHeliostats()[k]->CGetSubHeliostatVertexes(grid_verts[gi]);
  }
  for (int ti = 0; ti < a->n_ids; ++ti) {
    const int hid = a->ids[ti];
    Heliostat* h = s->getHeliostats()[hid];
    auto* g = static_cast<RectangleGrid*>(s->getGrids()[h->getBelongingGridId()]);
    const int rid = g->getBelongingReceiverIndex();
    Receiver* rc = s->getReceivers()[rid];
    const std::vector<float3>& verts = grid_verts[h->getBelongingGridId()];
    const HeliostatArgument arg(nullptr, nullptr, nullptr, 0, sub_begin_of(hid), h->getSubHelioSize());
    // QuasiMonteCarloRayTracer::rayTracing (QuasiMonteCarloRayTracer.cpp:58-60).
    float ratio = h->getPixelLength() / rc->getPixelLength();
    float factor = cfg->getDni() * ratio * ratio * cfg->getReflected_rate() / float(L);
    int2 src;
    float2 len;
    int n;
    lattice(h, src, len, n);
    // Facet centres/normals are evaluated only for the facets traced; the
    // flat-heliostat host function writes element f of full-size arrays.
    std::unique_ptr<float3[]> O(new float3[std::max(n, 1)]), N(new float3[std::max(n, 1)]);
    const bool flat = Heliostat_type(h) == 0;
    const int* off = a->offsets + a->offset_base[hid];
    const int2 res = rc->getResolution();
#pragma omp parallel
    {
      std::vector<double> img(total_pix, 0.0);
      double pw = 0.0;
      long long cnt[6] = {0};
#pragma omp for schedule(dynamic, 64)
      for (int f = 0; f < n; ++f) {
        if (a->facet_stride > 1 && f % a->facet_stride != a->facet_phase) continue;
        if (flat)
          host_map_microhelio_center_and_normal(f, O.get(), N.get(), h->getNormal(), h->getSize(),
                                                h->getRowAndColumn(), src, h->getPixelLength(), h->getGap(),
                                                h->getPosition(), (size_t)n);
        else
          facet(h, f, src, len, n, O[f], N[f]);
        const float3 origin = O[f];
        for (int l = a->light_begin; l < a->light_end; ++l) {
          ++cnt[0];
          int address = (off[f] + l) % P;
          float3 sample = make_float3(a->pool_dirs[3 * address], a->pool_dirs[3 * address + 1],
                                      a->pool_dirs[3 * address + 2]);
          float3 dir = global_func::local2world_rotate(sample, -sun_dir);
          int code;
          if (rectGridDDA::collision(origin, dir, *g, verts.data(), arg)) {
            code = -1;
            ++cnt[1];
          } else {
            address = (off[(f + 1) % P] + l) % P;
            float3 pert = make_float3(a->pool_pert[3 * address], a->pool_pert[3 * address + 1],
                                      a->pool_pert[3 * address + 2]);
            float3 normal = global_func::local2world_rotate(pert, N[f]);
            normal = normalize(normal);
            float3 rd = normalize(reflect(-dir, normal));
            if (rectGridDDA::collision(origin, rd, *g, verts.data(), arg)) {
              code = -2;
              ++cnt[2];
            } else {
              float t, u, v;
              bool hit = rc->getType() == 0 ? static_cast<RectangleReceiver*>(rc)->GIntersect(origin, rd, t, u, v)
                                            : static_cast<CylinderReceiver*>(rc)->GIntersect(origin, rd, t, u, v);
              if (!hit) {
                code = -3;
                ++cnt[3];
              } else {
                float energy = calEnergy(t, rd, normal, factor);
                int2 row_col = make_int2(u * res.y, v * res.x);
                if (row_col.x >= res.y || row_col.y >= res.x || row_col.x < 0 || row_col.y < 0) {
                  row_col.x = std::min(std::max(row_col.x, 0), res.y - 1);
                  row_col.y = std::min(std::max(row_col.y, 0), res.x - 1);
                  ++cnt[5];
                }
                code = row_col.x * res.x + row_col.y;
                ++cnt[4];
                if (a->images) img[a->image_base[rid] + code] += (double)energy;
                pw += (double)energy;
              }
            }
          }
          if (a->records && hid == a->rec_id && f >= a->rec_facet_begin && f < a->rec_facet_end)
            a->records[(long long)(f - a->rec_facet_begin) * (a->light_end - a->light_begin) + (l - a->light_begin)] = code;
        }
      }
#pragma omp critical
      {
        if (a->images)
          for (long long i = 0; i < total_pix; ++i) a->images[i] += img[i];
        if (a->power) a->power[hid] += pw;
        for (int k = 0; k < 6; ++k) totals[k] += cnt[k];
      }
    }
  }
  if (a->counters)
    for (int k = 0; k < 6; ++k) a->counters[k] += totals[k];
}

// trimmed_mean's loop (Tool/Smoother/ImageSmoother.cu:13-64) on the
// reference's own Max_heap / Min_heap (heap.cuh).
void ref_smooth(const float* in, float* out, int width, int height, int kernel_radius, float trimmed_ratio) {
  Quiet quiet;
  std::streambuf* old = std::cout.rdbuf(nullptr);
#pragma omp parallel for schedule(static)
  for (int y = 0; y < height; ++y) {
    int k0 = (2 * kernel_radius + 1) * (2 * kernel_radius + 1) * trimmed_ratio + 1;
    std::vector<float> sdata(2 * k0 + 2);
    for (int x = 0; x < width; ++x) {
      int2 lu = make_int2((x - kernel_radius >= 0) ? (x - kernel_radius) : 0,
                          (y - kernel_radius >= 0) ? (y - kernel_radius) : 0);
      int2 rb = make_int2((x + kernel_radius < width) ? (x + kernel_radius) : width - 1,
                          (y + kernel_radius < height) ? (y + kernel_radius) : height - 1);
      int cnt = (rb.x - lu.x + 1) * (rb.y - lu.y + 1);
      int k = cnt * trimmed_ratio;
      Max_heap max_heap(k, &sdata[0]);
      Min_heap min_heap(k, &sdata[k0]);
      float value = 0.0f;
      for (int r = lu.y; r <= rb.y; ++r)
        for (int c = lu.x; c <= rb.x; ++c) {
          float cur = in[(size_t)r * width + c];
          value += cur;
          if (!max_heap.full()) {
            max_heap.insert(cur);
            min_heap.insert(cur);
          } else if (cur < max_heap.top()) {
            max_heap.delete_and_insert(cur);
          } else if (cur > min_heap.top()) {
            min_heap.delete_and_insert(cur);
          }
        }
      out[(size_t)y * width + x] = (value - max_heap.sum() - min_heap.sum()) / float(cnt - 2 * k);
    }
  }
  std::cout.rdbuf(old);
}

// set_samplelights' table (Scene/SceneProcessor.cu:204-239) through the
// reference's parameters_generate; scalars5 = less_465, gamma, A, B, C.
void ref_buie_table(float csr, int num_group, float* cdf_x, float* cdf_y, float* kk, float* scalars5) {
  float upper_lm = 4.65f;
  float k = 0.9f * logf(13.5f * csr) * powf(csr, -0.3f);
  float gamma = 2.2f * logf(0.52f * csr) * powf(csr, 0.43f) - 0.1f;
  float i465 = samplelights::integration_larger_than_465_intensity(9.3f, k, gamma) -
               samplelights::integration_larger_than_465_intensity(upper_lm, k, gamma);
  std::vector<float> hk(num_group);
  float2* cdf = samplelights::parameters_generate(hk.data(), num_group, k, gamma, upper_lm);
  for (int i = 0; i <= num_group; ++i) cdf_x[i] = cdf[i].x, cdf_y[i] = cdf[i].y;
  for (int i = 0; i < num_group; ++i) kk[i] = hk[i];
  float less = cdf[num_group].y;
  scalars5[0] = less;
  scalars5[1] = gamma;
  scalars5[2] = less + i465;
  scalars5[3] = (gamma + 1) / expf(k);
  scalars5[4] = powf(upper_lm, gamma + 1);
  delete[] cdf;
}

// linear_interpolation's body (Scene/SceneProcessor.cu:61-81) over host uniforms.
void ref_buie_theta(float csr, int num_group, const float* uniforms, float* theta, int n) {
  std::vector<float> cx(num_group + 1), cy(num_group + 1), kk(num_group), sc(5);
  ref_buie_table(csr, num_group, cx.data(), cy.data(), kk.data(), sc.data());
  std::vector<float2> cdf(num_group + 1);
  for (int i = 0; i <= num_group; ++i) cdf[i] = make_float2(cx[i], cy[i]);
  const float less = sc[0], gamma = sc[1], A = sc[2], B = sc[3], C = sc[4];
  for (int i = 0; i < n; ++i) {
    float u = uniforms[i] * A;
    if (u < less) {
      int id = samplelights::max_less_index(cdf.data(), u, num_group);
      u = (u - cdf[id].y) * kk[id] + cdf[id].x;
      u = atan(sqrtf(u / 4.65f) * 0.5016916f);
    } else {
      u = powf((u - less) * B + C, 1 / (gamma + 1));
      float ri2 = 0.5016916f * 0.5016916f;
      float ro2 = 1.340874f * 1.340874f;
      u = atan(sqrt(ro2 + (u - 4.65f) / 4.65f * (ro2 - ri2)));
    }
    theta[i] = u / 100.0f;
  }
}

// TaskLoader::loadRayTracingHeliostatIndex on the loaded scene:
// 1 / 0, or -1 when it throws.  ids / grids in the reference's set order.
int ref_load_tasks(const char* path, int* ids, int* n_ids, int* grids, int* n_grids) {
  Quiet quiet;
  std::streambuf* old = std::cout.rdbuf(nullptr);
  int ans;
  try {
    ans = g_tasks.loadRayTracingHeliostatIndex(path, *SolarScene::GetInstance()) ? 1 : 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    ans = -1;
  }
  std::cout.rdbuf(old);
  if (ans >= 0) {
    int k = 0;
    for (int x : g_tasks.getHeliostatIndexesArray()) ids[k++] = x;
    *n_ids = k;
    k = 0;
    for (int x : g_tasks.getReceiverIndexesArray()) grids[k++] = x;
    *n_grids = k;
  }
  return ans;
}

// ImageSaver::saveText.
float ref_save_text(const char* path, int height, int width, float* data) {
  Quiet quiet;
  std::streambuf* old = std::cout.rdbuf(nullptr);
  float m = ImageSaver::saveText(path, height, width, data);
  std::cout.rdbuf(old);
  return m;
}

}  // extern "C"
