// CPU ORACLE HARNESS - test/benchmark infrastructure only.
//
// C entry points over the reference's own CUDA build (every .cu/.cpp of the
// reference tree except main.cpp and its tests, compiled by
// oracle/build_ref.py into oracle/_ref/libref_gpu.so with the real CUDA
// runtime and cuRAND).  bench.py uses it to time the reference's tracer on
// the same B200: QuasiMonteCarloRayTracer::rayTracing per heliostat, end to
// end (B1), and the map_raytracing launch alone (B2); tests/test_gpu_reference.py
// (through oracle/ref_gpu_parity.py) injects sample pools and facet offsets
// and compares the reference kernel's flux maps with this tracer's.
#include <cuda_runtime.h>

#include <cstdio>
#include <iostream>
#include <string>
#include <vector>

#define private public
#define protected public
#include "CylinderReceiver.cuh"
#include "CylinderReceiverRectangleGridRayTracing.cuh"
#include "QuasiMonteCarloRayTracer.h"
#include "RectangleGrid.cuh"
#include "RectangleReceiver.cuh"
#include "RectangleReceiverRectangleGridRayTracing.cuh"
#include "SceneConfiguration.h"
#include "SceneLoader.h"
#include "SceneProcessor.h"
#include "SolarScene.h"
#include "Grid/rectGridDDA.cuh"
#include "Receiver/receiverIntersectionUtil.cuh"
#include "global_function.cuh"
#undef private
#undef protected

namespace {
std::string g_err;
bool g_loaded = false;
}  // namespace

extern "C" {

const char* refgpu_last_error() { return g_err.c_str(); }

// Configuration + scene + SceneProcessor::processScene (cuRAND pools on the GPU).
int refgpu_load(const char* scene_path, const char* config_path, int* counts3) {
  if (g_loaded) {
    g_err = "the reference's singletons hold one scene per process";
    return -3;
  }
  try {
    SceneConfiguration* cfg = SceneConfiguration::getInstance();
    cfg->loadConfiguration(config_path);
    SolarScene* s = SolarScene::GetInstance();
    SceneLoader loader;
    if (!loader.SceneFileRead(s, scene_path)) {
      g_err = "SceneFileRead failed";
      return -2;
    }
    SceneProcessor proc(cfg);
    if (!proc.processScene(s)) {
      g_err = "processScene failed";
      return -2;
    }
    counts3[0] = (int)s->getReceivers().size();
    counts3[1] = (int)s->getGrids().size();
    counts3[2] = (int)s->getHeliostats().size();
    g_loaded = true;
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

// QuasiMonteCarloRayTracer::rayTracing for each listed heliostat, unchanged
// (its own cuRAND facet offsets, per-heliostat allocations and syncs); the
// device time of the whole loop in ms.
int refgpu_trace_pipeline(const int* ids, int n, float* ms) {
  try {
    SolarScene* s = SolarScene::GetInstance();
    QuasiMonteCarloRayTracer tracer;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaDeviceSynchronize();
    cudaEventRecord(a);
    for (int i = 0; i < n; ++i) tracer.rayTracing(s, ids[i]);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    cudaEventElapsedTime(ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return cudaGetLastError() == cudaSuccess ? 0 : -4;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

// The tracing launch alone: for each heliostat the reference's arguments are
// prepared (vertex table, micro-facets, offsets) outside the timed region,
// then only Rectangle/CylinderReceiverRectangleGridRayTracing is timed.
// Total kernel ms over the listed heliostats.
int refgpu_trace_kernels(const int* ids, int n, float* ms) {
  try {
    SolarScene* s = SolarScene::GetInstance();
    QuasiMonteCarloRayTracer tracer;
    Sunray* sun = s->getSunray();
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    float total = 0.0f;
    for (int i = 0; i < n; ++i) {
      const int id = ids[i];
      Heliostat* h = s->getHeliostats()[id];
      Grid* grid = s->getGrids()[h->getBelongingGridId()];
      Receiver* recv = s->getReceivers()[grid->getBelongingReceiverIndex()];
      float3* verts = nullptr;
      tracer.setFlatRectangleHeliostatVertexs(verts, s->getHeliostats(), grid->getStartHeliostatIndex(),
                                              grid->getStartHeliostatIndex() + grid->getNumberOfHeliostats());
      SunrayArgument sa = tracer.generateSunrayArgument(sun);
      HeliostatArgument ha = tracer.generateHeliostatArgument(s, id);
      float ratio = h->getPixelLength() / recv->getPixelLength();
      float factor = sun->getDNI() * ratio * ratio * sun->getReflectiveRate() / float(sun->getNumOfSunshapeLightsPerGroup());
      cudaDeviceSynchronize();
      cudaEventRecord(a);
      if (recv->getType() == 0)
        RectangleReceiverRectangleGridRayTracing(sa, dynamic_cast<RectangleReceiver*>(recv),
                                                 dynamic_cast<RectangleGrid*>(grid), ha, verts, factor);
      else
        CylinderReceiverRectangleGridRayTracing(sa, dynamic_cast<CylinderReceiver*>(recv),
                                                dynamic_cast<RectangleGrid*>(grid), ha, verts, factor);
      cudaEventRecord(b);
      cudaEventSynchronize(b);
      float t = 0.0f;
      cudaEventElapsedTime(&t, a, b);
      total += t;
      cudaFree(verts);
      ha.CClear();
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    *ms = total;
    return cudaGetLastError() == cudaSuccess ? 0 : -4;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

// Number of micro-facets of a heliostat: the host-side lattice arithmetic
// that opens CGetDiscreteMicroHelioOriginsAndNormals (RectangleHelio.cu:84-104,
// FocusFlatRectangleHelio.cu:68-82), without launching its kernels (the
// focus-flat ones read device frames that only exist after
// CGetSubHeliostatVertexes).
int refgpu_num_facets(int id) {
  Heliostat* h = SolarScene::GetInstance()->getHeliostats()[id];
  int2 rc = h->getRowAndColumn();
  float3 size = h->getSize();
  float2 gap = h->getGap();
  float lx = (size.z - gap.y * (rc.x - 1)) / float(rc.x);
  float ly = (size.x - gap.x * (rc.y - 1)) / float(rc.y);
  int sx = int(lx / h->getPixelLength());
  int sy = int(ly / h->getPixelLength());
  return rc.x * rc.y * sx * sy;
}

int refgpu_lights_per_group() { return SolarScene::GetInstance()->getSunray()->getNumOfSunshapeLightsPerGroup(); }

int refgpu_pool_size() {
  Sunray* sun = SolarScene::GetInstance()->getSunray();
  return sun->getNumOfSunshapeGroups() * sun->getNumOfSunshapeLightsPerGroup();
}

// Replaces the sun's sample pools after processScene, as the reference's
// own tests do (Sunray::CClear, then setDeviceSampleLights /
// setDevicePerturbation with new device arrays; receiverIntersectUtil.cpp:8-33).
int refgpu_set_pools(const float* dirs, const float* perturbations, int n) {
  Sunray* sun = SolarScene::GetInstance()->getSunray();
  if (n != sun->getNumOfSunshapeGroups() * sun->getNumOfSunshapeLightsPerGroup()) {
    g_err = "pool size differs from groups x lights per group";
    return -2;
  }
  sun->CClear();
  float3 *d_dirs = nullptr, *d_pert = nullptr;
  if (cudaMalloc(&d_dirs, sizeof(float3) * n) != cudaSuccess || cudaMalloc(&d_pert, sizeof(float3) * n) != cudaSuccess) {
    g_err = "cudaMalloc failed";
    return -4;
  }
  cudaMemcpy(d_dirs, dirs, sizeof(float3) * n, cudaMemcpyHostToDevice);
  cudaMemcpy(d_pert, perturbations, sizeof(float3) * n, cudaMemcpyHostToDevice);
  sun->setDeviceSampleLights(d_dirs);
  sun->setDevicePerturbation(d_pert);
  return cudaGetLastError() == cudaSuccess ? 0 : -4;
}

// The reference's tracing launch for one heliostat with the given facet
// offsets (num_facets + 1 entries: the launch reads entry f + 1 for facet f)
// in place of its cuRAND ones, accumulating into its receiver image: its
// vertex table, micro-facets and launcher unchanged.
int refgpu_trace_with_offsets(int id, const int* offsets, int n_offsets) {
  try {
    SolarScene* s = SolarScene::GetInstance();
    QuasiMonteCarloRayTracer tracer;
    Sunray* sun = s->getSunray();
    Heliostat* h = s->getHeliostats()[id];
    Grid* grid = s->getGrids()[h->getBelongingGridId()];
    Receiver* recv = s->getReceivers()[grid->getBelongingReceiverIndex()];
    float3* verts = nullptr;
    tracer.setFlatRectangleHeliostatVertexs(verts, s->getHeliostats(), grid->getStartHeliostatIndex(),
                                            grid->getStartHeliostatIndex() + grid->getNumberOfHeliostats());
    SunrayArgument sa = tracer.generateSunrayArgument(sun);
    HeliostatArgument ha = tracer.generateHeliostatArgument(s, id);
    if (n_offsets != ha.numberOfMicroHeliostats + 1) {
      cudaFree(verts);
      ha.CClear();
      g_err = "offsets must hold num_facets + 1 entries";
      return -2;
    }
    cudaFree(ha.d_microHelio_groups);
    ha.d_microHelio_groups = nullptr;
    cudaMalloc(&ha.d_microHelio_groups, sizeof(int) * n_offsets);
    cudaMemcpy(ha.d_microHelio_groups, offsets, sizeof(int) * n_offsets, cudaMemcpyHostToDevice);
    float ratio = h->getPixelLength() / recv->getPixelLength();
    float factor = sun->getDNI() * ratio * ratio * sun->getReflectiveRate() / float(sun->getNumOfSunshapeLightsPerGroup());
    if (recv->getType() == 0)
      RectangleReceiverRectangleGridRayTracing(sa, dynamic_cast<RectangleReceiver*>(recv),
                                               dynamic_cast<RectangleGrid*>(grid), ha, verts, factor);
    else
      CylinderReceiverRectangleGridRayTracing(sa, dynamic_cast<CylinderReceiver*>(recv),
                                              dynamic_cast<RectangleGrid*>(grid), ha, verts, factor);
    cudaDeviceSynchronize();
    cudaFree(verts);
    ha.CClear();
    return cudaGetLastError() == cudaSuccess ? 0 : -4;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

}  // extern "C"

namespace {

// Per-ray recorder of the reference's CUDA tracer: the steps of its
// map_raytracing kernels (CylinderReceiverRectangleGridRayTracing.cu:6-40,
// RectangleReceiverRectangleGridRayTracing.cu:6-41) for the rays of facets
// [facet_begin, facet_end) x every light index, calling the reference's own
// device functions (local2world_rotate, normalize, reflect,
// rectGridDDA::collision, the receiver's GIntersect, calEnergy), with the
// deposit (receiver_drawing's atomicAdd) replaced by a record per ray: the
// outcome code (pixel index row * width + col as receiver_drawing computes
// it, -1 shadowed, -2 blocked, -3 missed), u, v and the energy.
template <class Recv>
__global__ void record_rays(SunrayArgument sa, Recv recv, RectangleGrid grid, HeliostatArgument ha,
                            float3* verts, float factor, int facet_begin, int facet_end, int* codes, float* u_out,
                            float* v_out, float* energy) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int L = sa.numberOfLightsPerGroup;
  if (i >= (long long)(facet_end - facet_begin) * L) return;
  const long long ray = (long long)facet_begin * L + i;
  const long long f = ray / L;
  const int l = (int)(ray % L);
  int address = (ha.d_microHelio_groups[f] + l) % sa.pool_size;
  float3 dir = global_func::local2world_rotate(sa.d_samplelights[address], -sa.sunray_direction);
  const float3 origin = ha.d_microHelio_origins[f];
  int code = -1;
  float t = 0.0f, u = 0.0f, v = 0.0f, e = 0.0f;
  if (!rectGridDDA::collision(origin, dir, grid, verts, ha)) {
    float3 normal = ha.d_microHelio_normals[f];
    address = (ha.d_microHelio_groups[(f + 1) % sa.pool_size] + l) % sa.pool_size;
    normal = global_func::local2world_rotate(sa.d_perturbations[address], normal);
    normal = normalize(normal);
    dir = normalize(reflect(-dir, normal));
    if (rectGridDDA::collision(origin, dir, grid, verts, ha)) {
      code = -2;
    } else if (!recv.GIntersect(origin, dir, t, u, v)) {
      code = -3;
    } else {
      e = calEnergy(t, dir, normal, factor);
      const int2 res = recv.getResolution();
      const int2 row_col = make_int2(u * res.y, v * res.x);
      code = row_col.x * res.x + row_col.y;
    }
  }
  codes[i] = code;
  u_out[i] = u;
  v_out[i] = v;
  energy[i] = e;
}

}  // namespace

extern "C" {

// Records every ray of facets [facet_begin, facet_end) of one heliostat
// (all light indexes, row-major by facet) with the given facet offsets
// (num_facets + 1 entries): host output arrays of (facet_end - facet_begin)
// * lights entries each.  The reference's vertex table and micro-facets are
// built by its own code, as refgpu_trace_with_offsets does.
int refgpu_record_with_offsets(int id, const int* offsets, int n_offsets, int facet_begin, int facet_end,
                               int* codes, float* u, float* v, float* energy) {
  try {
    SolarScene* s = SolarScene::GetInstance();
    QuasiMonteCarloRayTracer tracer;
    Sunray* sun = s->getSunray();
    Heliostat* h = s->getHeliostats()[id];
    Grid* grid = s->getGrids()[h->getBelongingGridId()];
    Receiver* recv = s->getReceivers()[grid->getBelongingReceiverIndex()];
    float3* verts = nullptr;
    tracer.setFlatRectangleHeliostatVertexs(verts, s->getHeliostats(), grid->getStartHeliostatIndex(),
                                            grid->getStartHeliostatIndex() + grid->getNumberOfHeliostats());
    SunrayArgument sa = tracer.generateSunrayArgument(sun);
    HeliostatArgument ha = tracer.generateHeliostatArgument(s, id);
    if (n_offsets != ha.numberOfMicroHeliostats + 1 || facet_begin < 0 || facet_end > ha.numberOfMicroHeliostats ||
        facet_begin >= facet_end) {
      cudaFree(verts);
      ha.CClear();
      g_err = "offsets must hold num_facets + 1 entries and the facet range must lie inside the heliostat";
      return -2;
    }
    cudaFree(ha.d_microHelio_groups);
    ha.d_microHelio_groups = nullptr;
    cudaMalloc(&ha.d_microHelio_groups, sizeof(int) * n_offsets);
    cudaMemcpy(ha.d_microHelio_groups, offsets, sizeof(int) * n_offsets, cudaMemcpyHostToDevice);
    float ratio = h->getPixelLength() / recv->getPixelLength();
    float factor = sun->getDNI() * ratio * ratio * sun->getReflectiveRate() / float(sun->getNumOfSunshapeLightsPerGroup());
    const long long n = (long long)(facet_end - facet_begin) * sa.numberOfLightsPerGroup;
    int* d_codes = nullptr;
    float *d_u = nullptr, *d_v = nullptr, *d_e = nullptr;
    cudaMalloc(&d_codes, sizeof(int) * n);
    cudaMalloc(&d_u, sizeof(float) * n);
    cudaMalloc(&d_v, sizeof(float) * n);
    cudaMalloc(&d_e, sizeof(float) * n);
    const int threads = 256;
    const unsigned blocks = (unsigned)((n + threads - 1) / threads);
    if (recv->getType() == 0)
      record_rays<<<blocks, threads>>>(sa, *dynamic_cast<RectangleReceiver*>(recv), *dynamic_cast<RectangleGrid*>(grid),
                                       ha, verts, factor, facet_begin, facet_end, d_codes, d_u, d_v, d_e);
    else
      record_rays<<<blocks, threads>>>(sa, *dynamic_cast<CylinderReceiver*>(recv), *dynamic_cast<RectangleGrid*>(grid),
                                       ha, verts, factor, facet_begin, facet_end, d_codes, d_u, d_v, d_e);
    cudaError_t err = cudaDeviceSynchronize();
    if (err == cudaSuccess) err = cudaGetLastError();
    cudaMemcpy(codes, d_codes, sizeof(int) * n, cudaMemcpyDeviceToHost);
    cudaMemcpy(u, d_u, sizeof(float) * n, cudaMemcpyDeviceToHost);
    cudaMemcpy(v, d_v, sizeof(float) * n, cudaMemcpyDeviceToHost);
    cudaMemcpy(energy, d_e, sizeof(float) * n, cudaMemcpyDeviceToHost);
    cudaFree(d_codes);
    cudaFree(d_u);
    cudaFree(d_v);
    cudaFree(d_e);
    cudaFree(verts);
    ha.CClear();
    if (err != cudaSuccess) {
      g_err = cudaGetErrorString(err);
      return -4;
    }
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

int refgpu_clear_image(int r) {
  SolarScene::GetInstance()->getReceivers()[r]->Cclean_image_content();
  return cudaGetLastError() == cudaSuccess ? 0 : -4;
}

// Receiver image read-back (float, rows x cols).
int refgpu_image(int r, float* out, int* w, int* h) {
  Receiver* recv = SolarScene::GetInstance()->getReceivers()[r];
  *w = recv->getResolution().x;
  *h = recv->getResolution().y;
  if (out) cudaMemcpy(out, recv->getDeviceImage(), sizeof(float) * (*w) * (*h), cudaMemcpyDeviceToHost);
  return 0;
}

}  // extern "C"
