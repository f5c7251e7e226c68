// Host-side scene model: the reference's SolarScene contents after
// SceneLoader::SceneFileRead, SceneConfiguration::loadConfiguration and
// SceneProcessor::processScene, held as plain arrays.
//
// Everything here is float32 host arithmetic written in the reference's
// operation order (compiled with -ffp-contract=off), so the receiver
// vertices, heliostat normals, sub-heliostat vertex tables and grid cell
// lists equal what the reference builds on its host for the same files.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

namespace qm {

// Scene/SceneConfiguration.h:41-51 defaults; keys in Scene/SceneConfiguration.cpp:53-68.
struct SceneConfig {
  float3 sun_dir = {1.0f, 0.0f, 0.0f};
  float dni = 1000.0f;
  float csr = 0.1f;
  int num_sunshape_groups = 128;
  int num_per_sunshape_group = 2048;
  int inverse_transform_sampling_groups = 1024;
  float receiver_pixel_length = 0.01f;
  float helio_disturb_std = 0.001f;
  float helio_pixel_length = 0.01f;
  float helio_reflected_rate = 0.88f;
};

struct ReceiverModel {
  int type = 0;  // 0 rectangle, 1 cylinder
  float3 pos{}, size{}, normal{};
  int face = 0;
  // derived by init_receiver
  float pixel_length = 0.f;
  int2 resolution{0, 0};  // x = columns, y = rows
  float3 vertex[4]{};     // rectangle only
  float3 local_normal{};
  float3 focus{};         // rectangle only
};

struct GridModel {
  int type = 0;  // 0 = RectangleGrid
  float3 pos{}, size{}, interval{};
  int num_heliostats = 0;
  int heliostat_type = 0;
  int start_heliostat = 0;
  int receiver = 0;
  // derived by process_scene
  int3 cells{0, 0, 0};
  std::vector<int> cell_index;       // reference CSR: num_cells + 1 offsets
  std::vector<int> cell_match;       // reference CSR: sub-heliostat ids
  std::vector<int> cell_hindex;      // heliostat-level CSR offsets (same cells)
  std::vector<int> cell_hmatch;      // grid-local heliostat ids
  std::vector<float3> sub_vertices;  // 3 per sub-heliostat (reference vertex table)
  int num_subheliostats = 0;
};

struct HeliostatModel {
  int type = 0;  // 0 flat rectangle, 1 focus-flat rectangle
  float3 pos{}, size{};
  float2 gap{0.f, 0.f};
  int2 row_col{1, 1};
  float surface_property[6] = {-1, -1, -1, -1, -1, -1};
  int grid = 0;
  std::vector<float3> file_local_centers, file_local_normals;  // `subhelio` block
  // derived by process_scene
  float focus_length = -1.f;
  int read_method = -1;
  float pixel_length = 0.f;
  float3 focus{};                     // aim point on the receiver (sun-independent)
  float3 normal{};
  float3 vertex[4]{};
  int2 sub_row_col{0, 0};
  float2 sub_length{0.f, 0.f};       // x: along z (rows), y: along x (cols)
  int num_facets = 0;
  int num_sub = 1;
  int sub_begin = 0;                  // grid-local first sub-heliostat id
  std::vector<float3> local_centers;  // focus-flat: per sub-heliostat
  std::vector<float3> local_normals;
};

struct SceneModel {
  float ground_length = 0.f, ground_width = 0.f;
  int grid_num = 0;
  SceneConfig config;
  int config_fields = 0;
  std::vector<ReceiverModel> receivers;
  std::vector<GridModel> grids;
  std::vector<HeliostatModel> heliostats;
  bool processed = false;
};

// SceneLoader::SceneFileRead (Scene/SceneLoader.cpp:243-353).  Returns false
// and fills `err` where the reference prints to std::cerr and returns false.
bool read_scene_file(const std::string& path, SceneModel& scene, std::string& err);
bool read_scene_text(const std::string& text, SceneModel& scene, std::string& err);

// SceneConfiguration::loadConfiguration (Scene/SceneConfiguration.cpp:39-69).
// Returns the number of keys set, or -1 where the reference throws
// (missing file, malformed JSON).
int read_config_file(const std::string& path, SceneConfig& config, std::string& err);
int read_config_text(const std::string& text, SceneConfig& config, std::string& err);

// SceneProcessor::set_grid_receiver_heliostat_content
// (Scene/SceneProcessor.cpp:13-39) plus the per-trace vertex-table build of
// QuasiMonteCarloRayTracer::setFlatRectangleHeliostatVertexs
// (QuasiMonteCarloRayTracing/QuasiMonteCarloRayTracer.cpp:182-209).
bool process_scene(SceneModel& scene, std::string& err);

// Re-orients every heliostat of a processed scene toward a new sun direction
// (the sun-dependent half of process_scene: heliostat normals, corner
// vertices and sub-heliostat parallelograms; aim points, focus lengths, grid
// cell lists and facet counts do not depend on the sun).
void set_sun(SceneModel& scene, float3 sun_dir);

// TaskLoader::loadRayTracingHeliostatIndex (RayTracingPipeline/TaskLoader.cpp:114-204).
// Returns 1 (true), 0 (false: repeated or surplus indexes) or -1 where the
// reference throws.  `receivers` collects the grid id of each heliostat, as
// the reference does (TaskLoader.cpp:182), in first-seen order.
int read_task_file(const std::string& path, const SceneModel& scene, std::vector<int>& heliostats,
                   std::vector<int>& receivers, std::string& err);

// Facet lattice of one heliostat (RectangleHelio.cu:84-116 / FocusFlatRectangleHelio.cu:68-116).
void facet_lattice(const HeliostatModel& h, float pixel_length, int2& sub_row_col, float2& sub_length,
                   int& num_facets);

// ImageSaver::saveText (Tool/ImageSaver/ImageSaver.cpp:13-58): rows written top
// (highest row index) first, comma separated, values below 1e-5 as 0, fixed
// `precision` decimals.  Returns the maximum value written.
float save_text_image(const std::string& path, int height, int width, const float* data, int precision,
                      std::string& err, bool* ok);

}  // namespace qm
