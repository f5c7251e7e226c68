// Host program written against the reference's entry points, compiled
// against include/qmcrt_facade.hpp and linked with libqmcrt.so
// (tests/test_host.py, tests/test_gpu_parity.py).
//   facade_main <scene.scn> <config.json> <tasks.txt> <out_dir> <device>
// Prints one line of key=value results.
#include <cstdio>
#include <cstdlib>
#include <string>

#include "qmcrt_facade.hpp"

int main(int argc, char** argv) {
  if (argc != 6) return 2;
  const std::string scn = argv[1], cfg = argv[2], tasks = argv[3], out = argv[4];
  const int device = std::atoi(argv[5]);
  try {
    SceneConfiguration* config = SceneConfiguration::getInstance();
    const int fields = config->loadConfiguration(cfg);
    SolarScene* scene = SolarScene::GetInstance();
    scene->setDevice(device);
    SceneLoader loader;
    if (!loader.SceneFileRead(scene, scn)) return 3;
    SceneProcessor processor(config);
    if (!processor.processScene(scene)) return 4;
    TaskLoader task_loader;
    const bool tasks_ok = task_loader.loadRayTracingHeliostatIndex(tasks, *scene);
    double image_sum = -1.0;
    float saved_max = -1.0f;
    if (device >= 0) {
      QuasiMonteCarloRayTracer tracer;
      for (int id : task_loader.getHeliostatIndexesArray()) tracer.rayTracing(scene, id);
      int w = 0, h = 0;
      float* d_img = scene->receiverDeviceImage(0, &w, &h);
      std::vector<float> img = scene->receiverImage(0, &w, &h);
      image_sum = 0.0;
      for (float v : img) image_sum += v;
      ImageSmoother::image_smooth(d_img, 1, 0.17f, w, h);
      std::vector<float> smooth = scene->receiverImage(0, &w, &h);
      saved_max = ImageSaver::saveText(out + "/facade_after_smooth.txt", h, w, smooth.data());
    }
    std::printf("fields=%d heliostats=%d tasks_ok=%d tasks=%zu receivers=%zu image_sum=%.6e saved_max=%.6e\n", fields,
                scene->info().num_heliostats, tasks_ok ? 1 : 0, task_loader.getHeliostatIndexesArray().size(),
                task_loader.getReceiverIndexesArray().size(), image_sum, saved_max);
    scene->clear();
  } catch (const std::exception& e) {
    std::printf("error=%s\n", e.what());
    return 5;
  }
  return 0;
}
