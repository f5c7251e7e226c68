// Differentiable forward / adjoint pair (include/qmcrt.h, qmcrt_diff_*,
// qmcrt_fwd, qmcrt_bwd) over one scene at its current sun.
//
// The pair owns a one-instance batch (csrc/batch.cpp) whose preparation
// items carry the per-heliostat parameters, so the forward prepares the
// parameterised geometry on the device like any batch, traces with the
// bilinear-deposit output of the trace kernel (one hit bit per ray kept for
// the adjoint: hit records are checkpointed, 1 bit per ray, instead of
// re-walking the grid), smooths and evaluates the loss; the adjoint smooths
// the residual and runs the forward-mode kernel (csrc/diff.cu).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

#include "batch_state.h"
#include "diff.h"
#include "runtime.h"
#include "vecmath.h"

using namespace qrt;

struct qmcrt_diff {
  qmcrt_scene* scene = nullptr;
  qmcrt_batch* batch = nullptr;  // owned
  int H = 0;
  int radius = 0;
  std::vector<float> weights;
  DBuf d_weights, d_dtasks, d_bits, d_flux, d_tmp, d_target, d_resid, d_p, d_grad, d_loss, d_p_receivers;
  DBuf d_deposit;  // FP64 deposit of the forward, one double per image pixel
  std::vector<qm::DevReceiver> p_receivers;
  size_t image_floats = 0;
  bool forward_done = false;

  ~qmcrt_diff() {
    if (batch) {
      int prev = 0;
      cudaGetDevice(&prev);
      cudaSetDevice(batch->device);
      cudaDeviceSynchronize();
      for (DBuf* b : {&d_weights, &d_dtasks, &d_bits, &d_flux, &d_tmp, &d_target, &d_resid, &d_p, &d_grad, &d_loss,
                      &d_p_receivers, &d_deposit})
        b->release();
      cudaSetDevice(prev);
      qmcrt_batch_free(batch);
    }
  }
};

namespace {

qmcrt_diff* diff_checked(qmcrt_diff* d) {
  if (!d) invalid("differentiable context is NULL");
  return d;
}

// Aim axes of a heliostat on its receiver: for a cylinder the horizontal
// tangent at the aim point (the direction of increasing image column) and
// the vertical; for a rectangle its column and row edges.
void aim_axes(const qm::ReceiverModel& r, const qm::DevReceiver& dr, float3 focus, float3& au, float3& av) {
  if (r.type == 1) {
    float x = focus.x - r.pos.x, z = focus.z - r.pos.z;
    const float l = std::sqrt(x * x + z * z);
    if (l > 0.0f) {
      x /= l;
      z /= l;
      au = make_float3(-z, 0.0f, x);
    } else {
      au = make_float3(1.0f, 0.0f, 0.0f);
    }
    av = make_float3(0.0f, 1.0f, 0.0f);
  } else {
    au = qm::normalize(dr.ac);
    av = qm::normalize(dr.ab);
  }
}

}  // namespace

extern "C" {

int qmcrt_diff_create(qmcrt_scene* s, float sigma_px, qmcrt_diff** out) {
  return guarded([&] {
    if (!out) invalid("output handle is NULL");
    *out = nullptr;
    checked(s);
    if (!(sigma_px > 0.0f) || sigma_px > 64.0f) invalid("splat sigma must be in (0, 64] pixels");
    auto d = std::make_unique<qmcrt_diff>();
    d->scene = s;
    d->H = (int)s->model.heliostats.size();
    const int zero = 0;
    const float sun[3] = {s->model.config.sun_dir.x, s->model.config.sun_dir.y, s->model.config.sun_dir.z};
    qmcrt_scene* scenes[1] = {s};
    if (qmcrt_batch_create(scenes, 1, &zero, sun, 1, &d->batch) != QMCRT_OK)
      throw ApiError(QMCRT_ERR_CUDA, qmcrt_last_error());
    qmcrt_batch* b = d->batch;
    DeviceGuard guard(b->device);
    for (int h = 0; h < d->H; ++h) {
      const auto& hm = s->model.heliostats[h];
      const int r = s->model.grids[hm.grid].receiver;
      aim_axes(s->model.receivers[r], s->receivers[r], hm.focus, b->items[h].aim_u, b->items[h].aim_v);
    }
    d->radius = (int)std::ceil(3.0f * sigma_px);
    double sum = 0.0;
    std::vector<double> w(d->radius + 1);
    for (int k = 0; k <= d->radius; ++k) {
      w[k] = std::exp(-0.5 * k * k / ((double)sigma_px * sigma_px));
      sum += k == 0 ? w[k] : 2 * w[k];
    }
    for (double x : w) d->weights.push_back((float)(x / sum));
    upload(d->d_weights, d->weights);
    d->image_floats = b->d_images.bytes / sizeof(float);
    for (DBuf* x : {&d->d_flux, &d->d_tmp, &d->d_target, &d->d_resid, &d->d_p}) {
      x->alloc(d->image_floats * sizeof(float));
      cuda_check(cudaMemset(x->p, 0, x->bytes), "cudaMemset");
    }
    d->d_grad.alloc((size_t)std::max(d->H, 1) * qm::kDiffParams * sizeof(double));
    d->d_loss.alloc(sizeof(double));
    d->d_dtasks.alloc(b->tasks.size() * sizeof(qm::DiffTask));
    // The forward deposits into an FP64 image, rounded to the batch's float
    // image once per forward.
    d->d_deposit.alloc(d->image_floats * sizeof(double));
    for (size_t r = 0; r < b->receivers.size(); ++r) b->receivers[r].deposit = d->d_deposit.as<double>() + b->image_offset[r];
    upload(b->d_receivers, b->receivers);
    d->p_receivers = b->receivers;
    for (size_t r = 0; r < d->p_receivers.size(); ++r) d->p_receivers[r].image = d->d_p.as<float>() + b->image_offset[r];
    upload(d->d_p_receivers, d->p_receivers);
    *out = d.release();
  });
}

void qmcrt_diff_free(qmcrt_diff* d) { delete d; }

int qmcrt_diff_set_params(qmcrt_diff* d, const float* aim_offsets, const float* normal_offsets) {
  return guarded([&] {
    diff_checked(d);
    for (int h = 0; h < d->H; ++h) {
      qm::PrepItem& it = d->batch->items[h];
      it.aim_offset = aim_offsets ? make_float2(aim_offsets[2 * h], aim_offsets[2 * h + 1]) : make_float2(0.f, 0.f);
      it.normal_offset =
          normal_offsets ? make_float2(normal_offsets[2 * h], normal_offsets[2 * h + 1]) : make_float2(0.f, 0.f);
      if (!std::isfinite(it.aim_offset.x) || !std::isfinite(it.aim_offset.y) || !std::isfinite(it.normal_offset.x) ||
          !std::isfinite(it.normal_offset.y))
        invalid("parameters must be finite");
    }
    d->forward_done = false;
  });
}

int qmcrt_diff_set_target(qmcrt_diff* d, int receiver, const float* target) {
  return guarded([&] {
    diff_checked(d);
    qmcrt_batch* b = d->batch;
    if (receiver < 0 || receiver >= (int)b->receivers.size()) invalid("receiver index out of range");
    if (!target) invalid("target is NULL");
    const int2 shape = b->image_shape[receiver];
    DeviceGuard guard(b->device);
    cuda_check(cudaMemcpy(d->d_target.as<float>() + b->image_offset[receiver], target,
                          (size_t)shape.x * shape.y * sizeof(float), cudaMemcpyHostToDevice),
               "target upload");
    d->forward_done = false;
  });
}

int qmcrt_diff_set_light_range(qmcrt_diff* d, int begin, int end) {
  return guarded([&] {
    diff_checked(d);
    if (qmcrt_batch_set_light_range(d->batch, begin, end) != QMCRT_OK)
      throw ApiError(QMCRT_ERR_INVALID, qmcrt_last_error());
    d->forward_done = false;
  });
}

int qmcrt_fwd(qmcrt_diff* d, double* loss, void* stream) {
  return guarded([&] {
    diff_checked(d);
    qmcrt_batch* b = d->batch;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    DeviceGuard guard(b->device);
    batch_prepare(b, st);
    cuda_check(qm::launch_diff_prep(b->d_items.as<qm::PrepItem>(), (int)b->items.size(), b->d_tasks.as<qm::DevTask>(),
                                    d->d_dtasks.as<qm::DiffTask>(), st),
               "diff preparation");
    if (b->total_chunks < 0) batch_build_prefix(b);
    d->d_bits.alloc((size_t)std::max<long long>(b->total_chunks, 1) * 8 * sizeof(uint32_t));
    b->hit_bits = d->d_bits.as<uint32_t>();
    cuda_check(cudaMemsetAsync(d->d_deposit.p, 0, d->d_deposit.bytes, st), "clear");
    cuda_check(cudaMemsetAsync(b->d_power.p, 0, b->d_power.bytes, st), "clear");
    cuda_check(cudaMemsetAsync(d->d_loss.p, 0, sizeof(double), st), "clear");
    if (b->light_end > b->light_begin) cuda_check(batch_launch(b, st, 2), "forward trace");
    cuda_check(qm::launch_round_deposit(d->d_deposit.as<double>(), b->d_images.as<float>(), (long long)d->image_floats,
                                        st),
               "deposit rounding");
    for (size_t r = 0; r < b->receivers.size(); ++r) {
      const int2 sh = b->image_shape[r];
      const long long o = b->image_offset[r];
      cuda_check(qm::launch_gauss(b->d_images.as<float>() + o, d->d_tmp.as<float>() + o, d->d_flux.as<float>() + o, sh.x,
                                  sh.y, d->d_weights.as<float>(), d->radius, b->receivers[r].type == 1, st),
                 "splat smoothing");
      cuda_check(qm::launch_loss(d->d_flux.as<float>() + o, d->d_target.as<float>() + o, d->d_resid.as<float>() + o,
                                 (long long)sh.x * sh.y, d->d_loss.as<double>(), st),
                 "loss");
    }
    double L = 0.0;
    cuda_check(cudaMemcpyAsync(&L, d->d_loss.p, sizeof(double), cudaMemcpyDeviceToHost, st), "loss readback");
    cuda_check(cudaStreamSynchronize(st), "forward");
    if (loss) *loss = L;
    d->forward_done = true;
  });
}

int qmcrt_bwd(qmcrt_diff* d, double* grad, void* stream) {
  return guarded([&] {
    diff_checked(d);
    if (!d->forward_done) throw ApiError(QMCRT_ERR_STATE, "qmcrt_bwd needs a qmcrt_fwd with the current parameters");
    qmcrt_batch* b = d->batch;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    DeviceGuard guard(b->device);
    for (size_t r = 0; r < b->receivers.size(); ++r) {
      const int2 sh = b->image_shape[r];
      const long long o = b->image_offset[r];
      cuda_check(qm::launch_gauss(d->d_resid.as<float>() + o, d->d_tmp.as<float>() + o, d->d_p.as<float>() + o, sh.x,
                                  sh.y, d->d_weights.as<float>(), d->radius, b->receivers[r].type == 1, st),
                 "residual smoothing");
    }
    cuda_check(cudaMemsetAsync(d->d_grad.p, 0, d->d_grad.bytes, st), "clear");
    qm::BackwardParams p{};
    p.tasks = b->d_tasks.as<qm::DevTask>();
    p.dtasks = d->d_dtasks.as<qm::DiffTask>();
    p.receivers = d->d_p_receivers.as<qm::DevReceiver>();
    p.chunk_prefix = b->d_prefix.as<long long>();
    p.num_tasks = (int)b->tasks.size();
    p.total_chunks = b->total_chunks;
    p.light_begin = b->light_begin;
    p.light_end = b->light_end;
    p.hit_bits = d->d_bits.as<uint32_t>();
    p.grad = d->d_grad.as<double>();
    cuda_check(qm::launch_diff_backward(p, st), "adjoint kernel");
    if (grad)
      cuda_check(cudaMemcpyAsync(grad, d->d_grad.p, (size_t)d->H * qm::kDiffParams * sizeof(double),
                                 cudaMemcpyDeviceToHost, st),
                 "gradient readback");
    cuda_check(cudaStreamSynchronize(st), "adjoint");
  });
}

int qmcrt_diff_flux(qmcrt_diff* d, int receiver, float* out, int* width, int* height) {
  return guarded([&] {
    diff_checked(d);
    qmcrt_batch* b = d->batch;
    if (receiver < 0 || receiver >= (int)b->receivers.size()) invalid("receiver index out of range");
    const int2 sh = b->image_shape[receiver];
    if (width) *width = sh.x;
    if (height) *height = sh.y;
    if (!out) return;
    DeviceGuard guard(b->device);
    cuda_check(cudaMemcpy(out, d->d_flux.as<float>() + b->image_offset[receiver], (size_t)sh.x * sh.y * sizeof(float),
                          cudaMemcpyDeviceToHost),
               "flux readback");
  });
}

}  // extern "C"
