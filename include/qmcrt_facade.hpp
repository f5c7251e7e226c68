/*
 * qmcrt_facade.hpp - header-only C++ facade with the reference's class and
 * method names over the C ABI (qmcrt.h), so host code written against
 * SolarEnergy_Chier's entry points keeps its shape:
 *
 *   SceneConfiguration::getInstance()->loadConfiguration(path)   Scene/SceneConfiguration.h:13-14
 *   SceneLoader().SceneFileRead(SolarScene*, path)               Scene/SceneLoader.h:26
 *   SceneProcessor(SceneConfiguration*).processScene(SolarScene*) Scene/SceneProcessor.h:17
 *   SolarScene::GetInstance(), clear()                           Scene/SolarScene.h:35, SolarScene.cpp:31-46
 *   QuasiMonteCarloRayTracer().rayTracing(SolarScene*, id)        QuasiMonteCarloRayTracing/QuasiMonteCarloRayTracer.h:13
 *   ImageSmoother::image_smooth(d_array, radius, ratio, w, h)     Tool/Smoother/ImageSmoother.cuh:20
 *   ImageSaver::saveText(file, height, width, h_data, precision)  Tool/ImageSaver/ImageSaver.h:12
 *   TaskLoader().loadRayTracingHeliostatIndex(path, SolarScene&)  RayTracingPipeline/TaskLoader.h:18-21
 *   RayTracingPipeline::rayTracing(argc, argv)                    RayTracingPipeline/RayTracingPipeline.h:13
 *
 * Differences, all at the boundary: the scene is built when processScene
 * runs (the C ABI loads scene and configuration together); CUDA errors
 * throw std::runtime_error instead of exit(1); rayTracing enqueues on the
 * legacy default stream and the read-backs synchronise (the reference
 * synchronises after every heliostat).  The classes live in namespace
 * qmcrt_ref and are also brought to global scope unless
 * QMCRT_FACADE_NO_GLOBAL_NAMES is defined.  Link with -lqmcrt.
 */
#ifndef QMCRT_FACADE_HPP
#define QMCRT_FACADE_HPP

#include <iostream>
#include <stdexcept>
#include <string>
#include <unordered_set>
#include <vector>

#include "qmcrt.h"

namespace qmcrt_ref {

inline void qmcrt_ok(int rc) {
  if (rc != QMCRT_OK) throw std::runtime_error(qmcrt_last_error());
}

class SceneConfiguration {
 public:
  static SceneConfiguration* getInstance() {
    static SceneConfiguration instance;
    return &instance;
  }
  // Number of the 10 fields the file sets; throws if the file is missing or
  // malformed (SceneConfiguration.cpp:39-69).
  int loadConfiguration(const std::string& configuration_file_path) {
    int fields = 0;
    qmcrt_ok(qmcrt_config_check(configuration_file_path.c_str(), &fields));
    path_ = configuration_file_path;
    return fields;
  }
  const std::string& path() const { return path_; }

 private:
  std::string path_;
};

class SolarScene {
 public:
  static SolarScene* GetInstance() {
    static SolarScene instance;
    return &instance;
  }
  ~SolarScene() { clear(); }
  bool clear() {
    if (handle_) qmcrt_scene_free(handle_);
    handle_ = nullptr;
    return true;
  }
  // Device and seed used by processScene (device -1: host-only geometry).
  void setDevice(int device) { device_ = device; }
  void setSeed(unsigned seed) { seed_ = seed; }
  qmcrt_scene* handle() const { return handle_; }
  qmcrt_scene_info info() const {
    qmcrt_scene_info i{};
    qmcrt_ok(qmcrt_scene_get_info(require(), &i));
    return i;
  }
  // Receiver r's flux image (rows = height), read back from the device.
  std::vector<float> receiverImage(int r, int* width, int* height) const {
    qmcrt_ok(qmcrt_receiver_image(require(), r, nullptr, width, height));
    std::vector<float> out((size_t)*width * *height);
    qmcrt_ok(qmcrt_receiver_image(require(), r, out.data(), width, height));
    return out;
  }
  float* receiverDeviceImage(int r, int* width, int* height) const {
    float* p = nullptr;
    qmcrt_ok(qmcrt_receiver_device_image(require(), r, &p, width, height));
    return p;
  }
  // Receiver::Cclean_image_content (Receiver.cu:33-45).
  void cleanImage(int r) const { qmcrt_ok(qmcrt_receiver_clear(require(), r, nullptr)); }

 private:
  friend class SceneLoader;
  friend class SceneProcessor;
  qmcrt_scene* require() const {
    if (!handle_) throw std::runtime_error("the scene has not been processed (SceneProcessor::processScene)");
    return handle_;
  }
  std::string scene_path_;
  qmcrt_scene* handle_ = nullptr;
  int device_ = 0;
  unsigned seed_ = 0;
};

class SceneLoader {
 public:
  // Reads and checks the scene file against the loaded configuration (host
  // only); false with a message on std::cerr, as the reference.
  bool SceneFileRead(SolarScene* solarScene, const std::string& filepath) {
    const std::string& cfg = SceneConfiguration::getInstance()->path();
    if (cfg.empty()) {
      std::cerr << "SceneFileRead: load the configuration first" << std::endl;
      return false;
    }
    qmcrt_scene* probe = nullptr;
    if (qmcrt_scene_load(filepath.c_str(), cfg.c_str(), -1, 0u, &probe) != QMCRT_OK) {
      std::cerr << qmcrt_last_error() << std::endl;
      return false;
    }
    qmcrt_scene_free(probe);
    solarScene->scene_path_ = filepath;
    return true;
  }
};

class SceneProcessor {
 public:
  explicit SceneProcessor(SceneConfiguration* sceneConfiguration) : config_(sceneConfiguration) {}
  // Builds the scene on the device: geometry, grid cell lists, sample pools
  // and facet offsets (SceneProcessor.cpp:9-39, SceneProcessor.cu:147-271).
  bool processScene(SolarScene* solarScene) {
    solarScene->clear();
    qmcrt_scene* h = nullptr;
    if (qmcrt_scene_load(solarScene->scene_path_.c_str(), config_->path().c_str(), solarScene->device_,
                         solarScene->seed_, &h) != QMCRT_OK) {
      std::cerr << qmcrt_last_error() << std::endl;
      return false;
    }
    solarScene->handle_ = h;
    return true;
  }

 private:
  SceneConfiguration* config_;
};

class QuasiMonteCarloRayTracer {
 public:
  void rayTracing(SolarScene* solarScene, int heliostat_id) {
    qmcrt_ok(qmcrt_trace_heliostat(solarScene->handle(), heliostat_id, nullptr));
  }
};

class ImageSmoother {
 public:
  static void image_smooth(float* d_array, int kernel_radius, float trimmed_ratio, int width, int height) {
    qmcrt_ok(qmcrt_smooth(d_array, width, height, kernel_radius, trimmed_ratio, nullptr));
  }
};

class ImageSaver {
 public:
  static float saveText(const std::string& filename, int height, int width, const float* h_data, int precision = 2) {
    float max_value = 0.0f;
    qmcrt_ok(qmcrt_save_text(filename.c_str(), height, width, h_data, precision, &max_value));
    return max_value;
  }
};

class TaskLoader {
 public:
  bool loadRayTracingHeliostatIndex(const std::string& task_path, SolarScene& solarScene) {
    const int cap = solarScene.info().num_heliostats + 1;
    std::vector<int> h(cap), r(cap);
    int nh = 0, nr = 0, status = 0;
    qmcrt_ok(qmcrt_load_tasks(solarScene.handle(), task_path.c_str(), h.data(), &nh, cap, r.data(), &nr, &status));
    heliostat_indexes_ = std::unordered_set<int>(h.begin(), h.begin() + nh);
    receiver_indexes_ = std::unordered_set<int>(r.begin(), r.begin() + nr);
    return status == 1;
  }
  const std::unordered_set<int>& getHeliostatIndexesArray() const { return heliostat_indexes_; }
  const std::unordered_set<int>& getReceiverIndexesArray() const { return receiver_indexes_; }

 private:
  std::unordered_set<int> heliostat_indexes_, receiver_indexes_;
};

class RayTracingPipeline {
 public:
  static void rayTracing(int argc, char* argv[]) { qmcrt_ok(qmcrt_pipeline_run(argc, argv)); }
};

}  // namespace qmcrt_ref

#ifndef QMCRT_FACADE_NO_GLOBAL_NAMES
using qmcrt_ref::ImageSaver;
using qmcrt_ref::ImageSmoother;
using qmcrt_ref::QuasiMonteCarloRayTracer;
using qmcrt_ref::RayTracingPipeline;
using qmcrt_ref::SceneConfiguration;
using qmcrt_ref::SceneLoader;
using qmcrt_ref::SceneProcessor;
using qmcrt_ref::SolarScene;
using qmcrt_ref::TaskLoader;
#endif

#endif  // QMCRT_FACADE_HPP
