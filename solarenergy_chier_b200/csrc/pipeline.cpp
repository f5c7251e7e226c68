// RayTracingPipeline::rayTracing (RayTracingPipeline/RayTracingPipeline.cpp:16-142)
// on the C ABI: parse -c/-s/-o/-h, load and process the scene, load the task
// list, trace every listed heliostat in one launch, then for each recorded
// receiver index write the flux map before and after the trimmed-mean
// smoother (radius 5, ratio 0.05) and clear the image.
#include <getopt.h>
#include <sys/stat.h>

#include <chrono>
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

#include "qmcrt.h"

namespace {

struct Args {
  std::string config, scene, output, tasks;
};

// ArgumentParser::check_valid_file / check_valid_directory
// (Tool/ArgumentParser/ArgumentParser.cpp:21-46).
bool valid_file(const std::string& path, const std::string& suffix, std::string& err) {
  if (path.size() < suffix.size() || path.substr(path.size() - suffix.size()) != suffix) {
    err = "The path of file ' " + path + " ' does not consist of ' " + suffix + " ' suffix.";
    return false;
  }
  std::ifstream f(path.c_str());
  if (!f.good()) {
    err = "The file ' " + path + " ' couldn't be opened. Please check your file path.";
    return false;
  }
  return true;
}

bool valid_directory(const std::string& dir, std::string& err) {
  if (dir.empty() || dir.back() != '/') {
    err = "' " + dir + " ' directory format is incorrect. Please add '/' at the end of the path.";
    return false;
  }
  struct stat info {};
  if (stat(dir.c_str(), &info) != 0 || !S_ISDIR(info.st_mode)) {
    err = "' " + dir + " ' directory does not exist. Please check the path.";
    return false;
  }
  return true;
}

bool parse_args(int argc, char** argv, Args& a, std::string& err) {
  static struct option long_options[] = {{"configuration_path", required_argument, 0, 'c'},
                                         {"scene_path", required_argument, 0, 's'},
                                         {"output_path", required_argument, 0, 'o'},
                                         {"heliostat_index_path", required_argument, 0, 'h'},
                                         {0, 0, 0, 0}};
  optind = 1;
  int idx = 0, c;
  while ((c = getopt_long(argc, argv, "c:s:o:h:", long_options, &idx)) != -1) {
    if (c == 'c') a.config = optarg;
    else if (c == 's') a.scene = optarg;
    else if (c == 'o') a.output = optarg;
    else if (c == 'h') a.tasks = optarg;
    else {
      err = "Unknown arguments.";
      return false;
    }
  }
  return valid_file(a.config, ".json", err) && valid_file(a.scene, ".scn", err) &&
         valid_file(a.tasks, ".txt", err) && valid_directory(a.output, err);
}

int fail(const char* what) {
  std::fprintf(stderr, "%s: %s\n", what, qmcrt_last_error());
  return 1;
}

}  // namespace

extern "C" int qmcrt_pipeline_run(int argc, char** argv) {
  Args a;
  std::string err;
  if (!parse_args(argc, argv, a, err)) {
    std::fprintf(stderr, "%s\n", err.c_str());
    return 1;
  }
  qmcrt_scene* scene = nullptr;
  if (qmcrt_scene_load(a.scene.c_str(), a.config.c_str(), 0, 0u, &scene) != QMCRT_OK) return fail("scene");
  qmcrt_scene_info info;
  qmcrt_scene_get_info(scene, &info);
  std::vector<int> helios(info.num_heliostats + 1), recvs(info.num_heliostats + 1);
  int nh = 0, nr = 0, status = 0;
  if (qmcrt_load_tasks(scene, a.tasks.c_str(), helios.data(), &nh, (int)helios.size(), recvs.data(), &nr, &status) !=
      QMCRT_OK) {
    qmcrt_scene_free(scene);
    return fail("tasks");
  }
  if (status == 0) std::printf("Warning: the task list repeats or exceeds its heliostat count.\n");
  auto t0 = std::chrono::high_resolution_clock::now();
  if (qmcrt_trace_heliostats(scene, helios.data(), nh, nullptr) != QMCRT_OK) {
    qmcrt_scene_free(scene);
    return fail("trace");
  }
  double total_power = 0.0;
  if (qmcrt_power_fp64(scene, nullptr, &total_power) != QMCRT_OK) {  // synchronises the device
    qmcrt_scene_free(scene);
    return fail("trace");
  }
  auto t1 = std::chrono::high_resolution_clock::now();
  std::printf("Traced %d heliostat(s) in %lld microseconds; total power %.6f W.\n", nh,
              (long long)std::chrono::duration_cast<std::chrono::microseconds>(t1 - t0).count(), total_power);
  int w = 0, h = 0;
  std::vector<float> host;
  int rc = 0;
  for (int k = 0; k < nr; ++k) {
    // The reference records each heliostat's grid id as the receiver index
    // (RayTracingPipeline/TaskLoader.cpp:182) and saves that receiver.
    const int recv = recvs[k];
    if (recv < 0 || recv >= info.num_receivers) {
      std::fprintf(stderr, "receiver index %d (a grid id) has no receiver; skipped\n", recv);
      rc = 1;
      continue;
    }
    float* dimg = nullptr;
    qmcrt_receiver_device_image(scene, recv, &dimg, &w, &h);
    host.assign((size_t)w * h, 0.0f);
    if (qmcrt_receiver_image(scene, recv, host.data(), &w, &h) != QMCRT_OK) return fail("image");
    std::string base = a.output + std::to_string(recv);
    float mx = 0.0f;
    if (qmcrt_save_text((base + "_receiver_before_smooth.txt").c_str(), h, w, host.data(), 2, &mx) != QMCRT_OK)
      return fail("save");
    if (qmcrt_smooth(dimg, w, h, 5, 0.05f, nullptr) != QMCRT_OK) return fail("smooth");
    if (qmcrt_receiver_image(scene, recv, host.data(), &w, &h) != QMCRT_OK) return fail("image");
    if (qmcrt_save_text((base + "_receiver_after_smooth.txt").c_str(), h, w, host.data(), 2, &mx) != QMCRT_OK)
      return fail("save");
    std::printf("Receiver %d: max %.4f written to %s_receiver_{before,after}_smooth.txt\n", recv, mx, base.c_str());
    qmcrt_receiver_clear(scene, recv, nullptr);
  }
  qmcrt_scene_free(scene);
  return rc;
}
