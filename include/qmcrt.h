/*
 * qmcrt.h - C ABI of the B200 quasi-Monte-Carlo heliostat-field ray tracer.
 *
 * A drop-in for the QuasiMonteCarloRayTracer path of SolarEnergy_Chier: the
 * same .scn scene files, JSON configuration files and heliostat-index task
 * files, the same SolarScene / RayTracingPipeline steps, the same flux-map
 * text output.  Plain pointers and sizes only; every call returns a status
 * (QMCRT_OK or an error code) and qmcrt_last_error() gives the message of the
 * last failure on the calling thread.  No C++ exception crosses this
 * boundary.  Streams are passed as `void*` holding a cudaStream_t (NULL =
 * the legacy default stream).  A scene is owned by one host thread at a time.
 *
 * Each declaration names the reference interface it replaces
 * (file:line within the SolarEnergy_Chier tree).
 */
#ifndef QMCRT_H
#define QMCRT_H

#ifdef __cplusplus
extern "C" {
#endif

#define QMCRT_OK 0
#define QMCRT_ERR_INVALID 1   /* bad argument or index (reference: std::runtime_error)   */
#define QMCRT_ERR_IO 2        /* unreadable or malformed file (reference: false + cerr)  */
#define QMCRT_ERR_CUDA 3      /* CUDA runtime failure (reference: exit(1))               */
#define QMCRT_ERR_STATE 4     /* call out of order, e.g. no sample pool yet              */
#define QMCRT_ERR_NOMEM 5     /* device or host allocation failed (reference: exit(1))   */

typedef struct qmcrt_scene qmcrt_scene;

/* Message of the last failed call on this thread ("" when none). */
const char* qmcrt_last_error(void);
int qmcrt_version(void);

/* Fault injection for callers' error paths.  The reference has no
 * counterpart: it calls exit(1) when a CUDA allocation fails
 * (Util/check_cuda.h:18-27).  Every allocation this library makes for a
 * scene, batch or differentiable pair (device buffers, pinned staging, the
 * scene state) passes one gate; after `after` more allocations succeed the
 * next one fails with QMCRT_ERR_NOMEM and qmcrt_last_error() names it, as a
 * real out-of-memory does, and the injection disarms itself.  after < 0
 * disarms it.  The environment variable QMCRT_INJECT_ALLOC_FAILURE=<after>,
 * read when the library loads, arms it for programs that cannot call this
 * (e.g. bin/qmcrt).  Process-wide. */
int qmcrt_debug_fail_allocations(long long after);

/* ---- scene --------------------------------------------------------------
 * Replaces SceneConfiguration::getInstance()->loadConfiguration
 * (Scene/SceneConfiguration.cpp:39-69), SceneLoader::SceneFileRead
 * (Scene/SceneLoader.cpp:243-353) and the geometry half of
 * SceneProcessor::processScene (Scene/SceneProcessor.cpp:9-39): loads both
 * files, builds receivers, grid cell lists, heliostat normals and
 * sub-heliostat tables, and uploads them to `device`.  The sample pools and
 * facet offsets (the cuRAND half of processScene, Scene/SceneProcessor.cu:147-271
 * and Heliostat.cu:57-62) are generated with `seed` by the scrambled Sobol
 * generator; qmcrt_set_sample_pool / qmcrt_set_facet_offsets replace them.
 * device = -1 loads host-only: the processed geometry can be inspected with
 * the getters below on a machine without a GPU, every device call fails with
 * QMCRT_ERR_STATE. */
int qmcrt_scene_load(const char* scene_path, const char* config_path, int device, unsigned seed,
                     qmcrt_scene** out);
/* Replaces SolarScene::clear (Scene/SolarScene.cpp:31-46). */
void qmcrt_scene_free(qmcrt_scene* scene);
/* Replaces SceneConfiguration::loadConfiguration's parse alone
 * (Scene/SceneConfiguration.cpp:39-69): reads and checks a configuration
 * file; fields receives how many of the 10 keys it sets.  A missing or
 * malformed file is QMCRT_ERR_IO (the reference throws). */
int qmcrt_config_check(const char* config_path, int* fields);

/* New sun direction (direction of travel, as the configuration's "sun_dir").
 * Replaces reloading the configuration and re-running the sun-dependent half
 * of SceneProcessor::processScene (Scene/SceneProcessor.cpp:22-46:
 * Heliostat::CSetNormalAndRotate per heliostat and Sunray::setSunDirection):
 * heliostat normals, sub-heliostat parallelograms, traversal records and the
 * world-space sun-shape pool are rebuilt; pools, facet offsets, images and
 * powers are kept (clear them before tracing the new sun). */
int qmcrt_scene_set_sun(qmcrt_scene* scene, const float* sun_dir3);

typedef struct {
  int num_receivers, num_grids, num_heliostats;
  int num_sunshape_groups, num_per_sunshape_group, pool_size;
  int inverse_transform_sampling_groups, config_fields;
  float sun_dir[3];
  float dni, csr, receiver_pixel_length, helio_disturb_std, helio_pixel_length, helio_reflected_rate;
  float ground_length, ground_width;
  long long total_facets;
} qmcrt_scene_info;
/* SolarScene / SceneConfiguration getters (Scene/SolarScene.h:35-58, Scene/SceneConfiguration.h:20-33). */
int qmcrt_scene_get_info(const qmcrt_scene* scene, qmcrt_scene_info* info);

/* Receiver state after CInit (Scene/DataStructure/Receiver/Receiver.cuh:11-86):
 * vertices12 = 4 world vertices (rectangle), normal3 (normalised), focus3
 * (rectangle focus centre). */
int qmcrt_receiver_get(const qmcrt_scene* scene, int receiver, int* type, int* width, int* height,
                       float* pixel_length, float* vertices12, float* normal3, float* focus3);
/* Heliostat state after CSetNormalAndRotate (Scene/DataStructure/Heliostat/Heliostat.cuh:18-90). */
int qmcrt_heliostat_get(const qmcrt_scene* scene, int heliostat, int* type, int* grid, int* num_facets,
                        int* num_sub, int* sub_begin, float* pos3, float* size3, float* normal3,
                        float* focus_length);
/* Grid after Cinit + CGridHelioMatch (Scene/DataStructure/Grid/RectangleGrid.cu:8-117):
 * cells3, sub-heliostat count, CSR non-zeros, receiver, first heliostat, heliostat count. */
int qmcrt_grid_get(const qmcrt_scene* scene, int grid, int* cells3, int* num_sub, int* nnz, int* receiver,
                   int* start, int* count);
/* The grid's cell lists in the reference layout (d_grid_helio_index_,
 * d_grid_helio_match_; RectangleGrid.cuh:49-52): index has cells+1 entries. */
int qmcrt_grid_csr(const qmcrt_scene* scene, int grid, int* index, int* match);
/* Sub-heliostat vertex table of a grid, 9 floats per sub-heliostat
 * (QuasiMonteCarloRayTracer::setFlatRectangleHeliostatVertexs, QuasiMonteCarloRayTracer.cpp:182-209). */
int qmcrt_grid_vertices(const qmcrt_scene* scene, int grid, float* xyz);
/* Micro-facet centres and normals of a heliostat, 3 floats each, computed on
 * the device by the tracer's facet function (replaces
 * Heliostat::CGetDiscreteMicroHelioOriginsAndNormals, RectangleHelio.cu:84-116,
 * FocusFlatRectangleHelio.cu:68-116).  Host output buffers. */
int qmcrt_heliostat_facets(qmcrt_scene* scene, int heliostat, float* origins, float* normals);

/* ---- sampling ------------------------------------------------------------
 * Injection point for parity runs (the pool replacement of
 * Tests/QuasiMonteCarloRayTracingTests/receiverIntersectUtil.cpp:8-33):
 * dirs_xyz and perturb_xyz hold groups*per_group float3 each, host memory
 * (on_device = 0) or device memory (on_device = 1).  Every vector must be a
 * unit vector: one whose squared length lies outside [0.25, 4] (or is NaN)
 * is refused with QMCRT_ERR_INVALID and the scene keeps its pools (the
 * reference's pools are unit vectors by construction; the tracer normalises
 * the perturbed normal and the reflected ray without a range test). */
int qmcrt_set_sample_pool(qmcrt_scene* scene, const float* dirs_xyz, const float* perturb_xyz, int groups,
                          int per_group, int on_device);
/* Regenerates both pools on the device (replaces SceneProcessor::set_samplelights
 * and set_perturbation, Scene/SceneProcessor.cu:147-271).  sunshape 0 = Buie
 * from the configuration's csr (the reference's inverse CDF), 1 = pillbox of
 * half-angle `half_angle` radians.  Slope error sigma = helio_disturb_std. */
int qmcrt_generate_sample_pool(qmcrt_scene* scene, unsigned seed, int sunshape, float half_angle);
/* Reads back the pools (pool_size float3 each) into host buffers. */
int qmcrt_get_sample_pool(qmcrt_scene* scene, float* dirs_xyz, float* perturb_xyz);
/* Per-facet pool offsets of one heliostat (the d_microHelio_groups array,
 * Heliostat::generateDeviceMicrohelioGroup, Heliostat.cu:57-62).  n must be
 * num_facets (entry num_facets is then set to offsets[0]) or num_facets + 1
 * (the extra entry is what the reference's kernel reads for the last facet). */
int qmcrt_set_facet_offsets(qmcrt_scene* scene, int heliostat, const int* offsets, int n);
int qmcrt_get_facet_offsets(qmcrt_scene* scene, int heliostat, int* offsets, int n);
int qmcrt_generate_facet_offsets(qmcrt_scene* scene, unsigned seed);

/* exact = 1 selects the kernel build without FMA contraction (every float
 * operation rounded as the CPU oracle rounds it); 0 (default) the production
 * build (one-warp blocks, 72 registers per thread, 28 blocks per SM); 2
 * the production build in 256-thread blocks at 64 registers (four per SM);
 * 3 the production build with approximate per-ray arithmetic after the
 * shadow test (FMA contraction, hardware reciprocal square root and
 * approximate divisions in the slope-error normal, reflection, receiver test
 * and energy: hits near a pixel boundary or the cylinder's silhouette can
 * land one pixel over or flip, as in the reference's own CUDA build); 4 the
 * production build with only the arithmetic after the receiver's decisions
 * approximated (hit point, pixel position, energy): decisions as mode 0,
 * hits within a few ulp of a pixel edge one pixel over. */
int qmcrt_set_math_mode(qmcrt_scene* scene, int exact);
/* Launch shapes of the production build (math mode 0), indexes 0..count-1:
 * threads per block, warp-chunk iterations (32 rays each) and whether the
 * launch is persistent (a grid of resident warps taking warp chunks from a
 * work counter, instead of one warp per chunk); shape 0 is the default.  No
 * reference counterpart: the reference launches 512-thread blocks of one
 * ray each (Util/global_function.cuh:159-197).  Any array may be NULL; at
 * most 16 shapes. */
int qmcrt_launch_shapes(int* threads, int* chunk_iters, int* persistent, int* count);
int qmcrt_set_launch_shape(qmcrt_scene* scene, int shape);
/* Autotuner: traces heliostats[0..n) over the current light range once per
 * launch shape of the production build (after one warm-up each), keeps the
 * fastest for the scene's flux launches and reports it (best) and every
 * shape's device time in ms (ms_per_shape, may be NULL).  Images and powers
 * are cleared after.  The scene must be in math mode 0. */
int qmcrt_autotune(qmcrt_scene* scene, const int* heliostats, int n, void* stream, int* best, float* ms_per_shape);
/* Trace only light indexes [begin, end) of every facet (default [0, per_group)).
 * Energies keep the full-trace factor DNI*(hpx/rpx)^2*rho/per_group. */
int qmcrt_set_light_range(qmcrt_scene* scene, int begin, int end);

/* ---- tracing -------------------------------------------------------------
 * Replaces QuasiMonteCarloRayTracer::rayTracing(SolarScene*, int)
 * (QuasiMonteCarloRayTracing/QuasiMonteCarloRayTracer.cpp:15-91): adds the
 * heliostat's flux into its receiver's image (images accumulate until
 * cleared) and its FP64 power into the per-heliostat total.  Asynchronous on
 * `stream`.  Invalid indexes fail as checkValidHeliostatIndex (:96-127) does. */
int qmcrt_trace_heliostat(qmcrt_scene* scene, int heliostat, void* stream);
/* All listed heliostats in one launch (the loop of RayTracingPipeline.cpp:66-81). */
int qmcrt_trace_heliostats(qmcrt_scene* scene, const int* heliostats, int n, void* stream);

/* Receiver image, resolution.y rows of resolution.x floats
 * (Receiver::getDeviceImage, Receiver.cuh:69-75).  `out` is host memory;
 * the call synchronises the scene's device. */
int qmcrt_receiver_image(qmcrt_scene* scene, int receiver, float* out, int* width, int* height);
int qmcrt_receiver_device_image(qmcrt_scene* scene, int receiver, float** device_ptr, int* width, int* height);
/* Replaces Receiver::Cclean_image_content (Scene/DataStructure/Receiver/Receiver.cu:33-45). */
int qmcrt_receiver_clear(qmcrt_scene* scene, int receiver, void* stream);
/* FP64 per-heliostat energy and total accumulated by the tracer since the
 * last qmcrt_power_clear (per_heliostat: num_heliostats doubles, may be NULL). */
int qmcrt_power_fp64(qmcrt_scene* scene, double* per_heliostat, double* total);
int qmcrt_power_clear(qmcrt_scene* scene);
/* Counters: [0] receiver hits clamped into the image (u or v == 1),
 * [1] grid walks stopped by the step bound, [2..3] reserved. */
int qmcrt_diagnostics(qmcrt_scene* scene, unsigned long long* out4);

/* Rebuilds a grid's device cell lists on the GPU (count, scan, fill and
 * sort kernels) instead of from the host's lists: the same lists as
 * RectangleGrid::CGridHelioMatch builds (Scene/DataStructure/Grid/RectangleGrid.cu:62-117),
 * every heliostat in every cell its box pos +- |size|/2 covers, in
 * heliostat order.  The lists are replaced in place, so batches sharing
 * them stay valid; call it with no trace of the scene in flight.  ms
 * receives the device time of the build (may be NULL). */
int qmcrt_grid_build_device(qmcrt_scene* scene, int grid, float* ms);
/* Debug: the device cell lists of a grid: ranges (2 ints per cell,
 * [begin, end)), entries (4 ints each: heliostat, first sub-heliostat,
 * count, 0) and their number (either array may be NULL). */
int qmcrt_debug_grid_cells(qmcrt_scene* scene, int grid, int* ranges, int* entries, long long* num_entries);
/* Debug: per heliostat, the shadow-walk code for the current sun and pool:
 * 1 when the tracer skips its shadow walks because no other heliostat can
 * shadow any of its rays (a conservative capsule test around the sun-shape
 * cone; no reference counterpart -- the reference walks every ray), k + 1
 * when only k (<= 6) listed heliostats can (a ray whose path meets none of
 * their padded boxes skips its walk), 0 when every ray walks. */
int qmcrt_debug_shadow_free(qmcrt_scene* scene, int* flags);
/* Debug: per sub-heliostat of a grid (grid-local ids, as qmcrt_grid_vertices),
 * the block-walk code of its facets for the current sun and pools: 1 when
 * the walks are skipped because no other heliostat can block a ray
 * reflected from it (same kind of test around its reflected cone), k + 1
 * when only k (<= 6) listed heliostats can (a ray whose path meets none of
 * their padded boxes skips its walk), 0 when every ray walks. */
int qmcrt_debug_block_free(qmcrt_scene* scene, int grid, int* flags);

/* Per-ray outcome for facets [facet_begin, facet_end) x lights [light_begin,
 * light_end) of one heliostat, row-major by facet: pixel index for a
 * receiver hit, -1 shadowed, -2 blocked, -3 missed the receiver.  Traces into
 * scratch; scene images and powers are untouched. */
int qmcrt_debug_hit_records(qmcrt_scene* scene, int heliostat, int facet_begin, int facet_end,
                            int light_begin, int light_end, int* codes);

/* Debug: one hit bit per ray of heliostats ids[0..n) over the scene's light
 * range, traced by the current math mode with nothing deposited (no
 * reference counterpart: the reference keeps no per-ray record).  Word w,
 * bit i is ray (w / C) * 32 C + (w % C) * 32 + i of the launch's rays, with
 * C = the tracer's warp-chunk iterations and rays numbered task by task, each
 * task's rays padded to whole chunks of 32 C (facet-major, lights fastest);
 * the layout depends only on the heliostat list and the light range, so two
 * math modes' bit arrays compare ray by ray.  words receives the number of
 * 32-bit words the launch needs; device_bits (device memory, capacity words;
 * NULL = only report words) is cleared and filled. */
int qmcrt_debug_hit_bits(qmcrt_scene* scene, const int* heliostats, int n, unsigned* device_bits,
                         long long capacity, long long* words, void* stream);

/* ---- batched tracing ------------------------------------------------------
 * No single reference counterpart: the reference traces one sun per
 * processed scene, one heliostat per QuasiMonteCarloRayTracer::rayTracing
 * call (QuasiMonteCarloRayTracer.cpp:15-91), looped by RayTracingPipeline
 * (RayTracingPipeline.cpp:66-81).  A batch holds n instances, each a
 * (scene, sun direction) pair with its own receiver images and FP64
 * per-heliostat powers; the sun-dependent half of SceneProcessor::processScene
 * (Scene/SceneProcessor.cpp:22-46) runs on the device for all instances, and
 * qmcrt_batch_trace traces every heliostat of every instance in one launch.
 * Instances share their scene's grid cell lists, sample pools and facet
 * offsets (as read when the batch is created or its suns are set); scenes
 * must outlive the batch and live on one device.  Light ranges are common to
 * all instances (at most the smallest lights-per-group of the scenes). */
typedef struct qmcrt_batch qmcrt_batch;
int qmcrt_batch_create(qmcrt_scene* const* scenes, int n_scenes, const int* scene_of_instance,
                       const float* sun_dirs3, int n_instances, qmcrt_batch** out);
void qmcrt_batch_free(qmcrt_batch* batch);
/* New sun directions (3 floats per instance), prepared on the device. */
int qmcrt_batch_set_suns(qmcrt_batch* batch, const float* sun_dirs3, void* stream);
int qmcrt_batch_set_light_range(qmcrt_batch* batch, int begin, int end);
int qmcrt_batch_set_math_mode(qmcrt_batch* batch, int mode);
int qmcrt_batch_info(const qmcrt_batch* batch, int* instances, int* tasks, long long* rays_per_trace);
int qmcrt_batch_trace(qmcrt_batch* batch, void* stream);
/* Captures (optionally a clear of images and powers, then) one trace into a
 * CUDA graph; qmcrt_batch_graph_launch replays it.  Changing the light range
 * or math mode drops the graph. */
int qmcrt_batch_capture_graph(qmcrt_batch* batch, int clear_first);
int qmcrt_batch_graph_launch(qmcrt_batch* batch, void* stream);
int qmcrt_batch_clear(qmcrt_batch* batch, void* stream);
int qmcrt_batch_image(qmcrt_batch* batch, int instance, int receiver, float* out, int* width, int* height);
int qmcrt_batch_power_fp64(qmcrt_batch* batch, int instance, double* per_heliostat, double* total);
/* Autotuner over the production build's launch shapes (qmcrt_launch_shapes;
 * identical per-ray arithmetic, so identical results up to the order of
 * float additions): times each on this batch, keeps the fastest in math mode
 * 0 and reports its index; ms_per_shape (may be NULL) receives every
 * shape's time.  Images and powers are cleared after.  qmcrt_batch_autotune
 * is the same with only the chosen shape's time. */
int qmcrt_batch_autotune_shapes(qmcrt_batch* batch, void* stream, int* chosen_shape, float* ms_per_shape);
int qmcrt_batch_autotune(qmcrt_batch* batch, void* stream, int* chosen_shape, float* ms);
int qmcrt_batch_set_launch_shape(qmcrt_batch* batch, int shape);
/* Debug: the device-prepared sub-heliostat vertices (B, A, C per
 * sub-heliostat, as qmcrt_grid_vertices) of one instance-grid and the
 * heliostat normals of one instance (either output may be NULL). */
int qmcrt_batch_debug_geometry(qmcrt_batch* batch, int instance, int grid, float* vertices, float* normals);

/* ---- differentiation ------------------------------------------------------
 * No reference counterpart (the reference has no derivative of its tracer).
 * A forward / adjoint pair over one scene at its current sun.  Parameters
 * per heliostat h: aim offset (du, dv) in metres along the receiver's aim
 * axes at the heliostat's aim point (cylinder: horizontal tangent and
 * vertical; rectangle: its column and row edges) and normal offset (a, b)
 * in radians about the u and v axes of the normal's frame.  The forward
 * traces every heliostat with its parameters (sun shape, slope error,
 * shadowing and blocking as the plain path), deposits each hit bilinearly at
 * its pixel position, smooths with a normalised Gaussian of sigma_px pixels
 * (flux F) and returns L = sum over pixels (F - target)^2 (FP64).  The adjoint
 * returns dL/d(parameters), 4 doubles per heliostat (du, dv, a, b), from a
 * hand-written forward-mode kernel along each hit ray, with shadowing and
 * blocking indicators detached and the receiver's edges treated by band
 * estimates of their boundary terms; hit records of the forward are kept
 * (1 bit per ray).  Common random numbers: the scene's pools and facet
 * offsets are reused by every forward. */
typedef struct qmcrt_diff qmcrt_diff;
int qmcrt_diff_create(qmcrt_scene* scene, float sigma_px, qmcrt_diff** out);
/* The pair over n_suns suns of one scene (sun_dirs: 3 floats each, direction
 * of travel), traced by one launch.  The parameters are shared by every sun
 * (each heliostat has one aim point and one normal offset); receiver indexes
 * of the target / flux / image calls run over the suns' receivers
 * (k x num_receivers + r for receiver r at sun k); the loss sums over all;
 * qmcrt_bwd and qmcrt_diff_power sum over the suns per heliostat. */
int qmcrt_diff_create_suns(qmcrt_scene* scene, const float* sun_dirs, int n_suns, float sigma_px, qmcrt_diff** out);
void qmcrt_diff_free(qmcrt_diff* diff);
/* Hit records of the forward for the adjoint: mode 0 chooses (checkpoint
 * while rays / 8 bytes fit in a quarter of the free device memory, else
 * recompute), 1 checkpoints them, 2 recomputes them in the adjoint with a
 * hit-bit trace of each segment of segment_rays rays (0 keeps the current
 * size; default 2^28 rays) before its adjoint launch.  Both give the same
 * gradient.  qmcrt_diff_hit_records reports the last forward's choice and
 * the checkpoint's size. */
int qmcrt_diff_set_hit_records(qmcrt_diff* diff, int mode, long long segment_rays);
int qmcrt_diff_hit_records(qmcrt_diff* diff, int* recomputed, long long* checkpoint_bytes);
/* aim_offsets, normal_offsets: 2 floats per heliostat each (NULL = zeros). */
int qmcrt_diff_set_params(qmcrt_diff* diff, const float* aim_offsets, const float* normal_offsets);
int qmcrt_diff_set_target(qmcrt_diff* diff, int receiver, const float* target);
int qmcrt_diff_set_light_range(qmcrt_diff* diff, int begin, int end);
int qmcrt_fwd(qmcrt_diff* diff, double* loss, void* stream);
int qmcrt_bwd(qmcrt_diff* diff, double* grad, void* stream);
/* The smoothed flux F of the last forward. */
int qmcrt_diff_flux(qmcrt_diff* diff, int receiver, float* out, int* width, int* height);
/* The plain tracer on the pair's current parameters: the same rays as the
 * forward, each hit's energy added to its nearest pixel (as
 * qmcrt_trace_heliostats), into the images and powers that qmcrt_diff_image
 * and qmcrt_diff_power read.  A pending qmcrt_bwd stays valid.  Used to check
 * an optimisation step against the tracer the reference runs. */
int qmcrt_diff_plain(qmcrt_diff* diff, void* stream);
/* Unsmoothed flux of the last trace: after qmcrt_fwd the bilinear deposit
 * (FP64, rounded to float), after qmcrt_diff_plain the plain flux. */
int qmcrt_diff_image(qmcrt_diff* diff, int receiver, float* out, int* width, int* height);
/* FP64 per-heliostat powers and their compensated total of the last trace
 * (forward or plain; equal up to summation order for the same parameters). */
int qmcrt_diff_power(qmcrt_diff* diff, double* per_heliostat, double* total);

/* ---- smoothing and output ------------------------------------------------
 * Replaces ImageSmoother::image_smooth (Tool/Smoother/ImageSmoother.cu:68-113):
 * in-place trimmed mean of a device image.  0 <= trim_ratio < 0.5. */
int qmcrt_smooth(float* device_image, int width, int height, int radius, float trim_ratio, void* stream);

/* No counterpart in the reference.  qmcrt_smooth without any device
 * allocation, for callers that may not call cudaMalloc (a fixed device-memory
 * budget already reserved by another allocator, or a real-time loop that
 * cannot take an allocation's latency or failure).  The image copy lives in a
 * static device array of 4,194,304 floats (16 MiB) that every GPU loading the
 * library holds until exit; larger images fail with QMCRT_ERR_INVALID.  The
 * first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) with that device current; make it before any stream
 * capture.  The address is kept for the life of the process: after
 * cudaDeviceReset (or any teardown of the device's primary context) the
 * module is loaded again and the kept address is stale, so do not call this
 * function on a device that has been reset.  All calls share the array:
 * calls that overlap on the GPU race. */
int qmcrt_smooth_static(float* device_image, int width, int height, int radius, float trim_ratio, void* stream);

/* Replaces TaskLoader::loadRayTracingHeliostatIndex (RayTracingPipeline/TaskLoader.cpp:114-204).
 * status: 1 true, 0 false (repeated or surplus indexes).  receivers receives the
 * grid ids of the listed heliostats, as the reference records them. */
int qmcrt_load_tasks(const qmcrt_scene* scene, const char* path, int* heliostats, int* num_heliostats,
                     int capacity, int* receivers, int* num_receivers, int* status);

/* Replaces ImageSaver::saveText (Tool/ImageSaver/ImageSaver.cpp:13-58). */
int qmcrt_save_text(const char* path, int height, int width, const float* host_data, int precision,
                    float* max_value);

/* Replaces RayTracingPipeline::rayTracing(argc, argv) (RayTracingPipeline/RayTracingPipeline.cpp:16-114),
 * getopt flags -c -s -o -h (Tool/ArgumentParser/ArgumentParser.cpp:49-94). */
int qmcrt_pipeline_run(int argc, char** argv);

#ifdef __cplusplus
}
#endif

#endif /* QMCRT_H */
