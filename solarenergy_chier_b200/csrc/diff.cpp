// Differentiable forward / adjoint pair (include/qmcrt.h, qmcrt_diff_*,
// qmcrt_fwd, qmcrt_bwd) over one scene at one or several suns.
//
// The pair owns a batch (csrc/batch.cpp) with one instance per sun, whose
// preparation items carry the per-heliostat parameters (shared by every
// sun: they are the heliostats' physical aim points and normal offsets), so
// the forward prepares the parameterised geometry on the device like any
// batch, traces with the bilinear-deposit output of the trace kernel,
// smooths and evaluates the loss summed over all suns' images; the adjoint
// smooths the residual and runs the forward-mode kernel (csrc/diff.cu), and
// the per-(sun, heliostat) gradients are summed per heliostat.
//
// Hit records (1 bit per ray: did the ray reach the receiver past shadowing
// and blocking) are either checkpointed by the forward or recomputed by the
// adjoint, segment by segment of warp chunks, with a hit-bit-only trace
// launch before each adjoint launch: checkpointing costs rays / 8 bytes,
// recomputing one more trace of every ray.  The automatic choice
// checkpoints while the bits take at most a quarter of the free device
// memory.
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
  int suns = 1;
  int hit_mode = 0;                       // 0 automatic, 1 checkpoint, 2 recompute
  long long segment_chunks = (1LL << 28) / qm::kChunk;  // warp chunks per recompute segment (2^28 rays)
  bool recompute = false;                 // the last forward's choice
  size_t n_slots = 0;                     // power slots of the batch (suns x heliostats)
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

}  // extern "C"

namespace {

void diff_create(qmcrt_scene* s, const float* sun_dirs, int n_suns, float sigma_px, qmcrt_diff** out) {
  if (!out) invalid("output handle is NULL");
  *out = nullptr;
  checked(s);
  if (!(sigma_px > 0.0f) || sigma_px > 64.0f) invalid("splat sigma must be in (0, 64] pixels");
  if (n_suns < 1) invalid("at least one sun is needed");
  auto d = std::make_unique<qmcrt_diff>();
  d->scene = s;
  d->H = (int)s->model.heliostats.size();
  d->suns = n_suns;
  std::vector<qmcrt_scene*> scenes{s};
  std::vector<int> scene_of(n_suns, 0);
  if (qmcrt_batch_create(scenes.data(), 1, scene_of.data(), sun_dirs, n_suns, &d->batch) != QMCRT_OK)
    throw ApiError(QMCRT_ERR_INVALID, qmcrt_last_error());
  qmcrt_batch* b = d->batch;
  DeviceGuard guard(b->device);
  for (const auto& I : b->inst) {
    for (int h = 0; h < d->H; ++h) {
      const auto& hm = s->model.heliostats[h];
      const int r = s->model.grids[hm.grid].receiver;
      aim_axes(s->model.receivers[r], s->receivers[r], hm.focus, b->items[I.task_base + h].aim_u,
               b->items[I.task_base + h].aim_v);
    }
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
  d->n_slots = b->d_power.bytes / sizeof(double);
  d->d_grad.alloc(std::max<size_t>(d->n_slots, 1) * qm::kDiffParams * sizeof(double));
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
}

// Per-heliostat sums over the suns of per-(sun, heliostat) slot values
// (FP64, in sun order).
std::vector<double> per_heliostat(const qmcrt_diff* d, const std::vector<double>& slots, int width) {
  std::vector<double> out((size_t)d->H * width, 0.0);
  for (const auto& I : d->batch->inst)
    for (int h = 0; h < d->H; ++h)
      for (int k = 0; k < width; ++k) out[(size_t)h * width + k] += slots[((size_t)I.power_base + h) * width + k];
  return out;
}

void check_receiver(const qmcrt_diff* d, int receiver) {
  if (receiver < 0 || receiver >= (int)d->batch->receivers.size())
    invalid("receiver index out of range (sun k, receiver r: k x receivers + r)");
}

}  // namespace

extern "C" {

int qmcrt_diff_create(qmcrt_scene* s, float sigma_px, qmcrt_diff** out) {
  return guarded([&] {
    checked(s);
    const float sun[3] = {s->model.config.sun_dir.x, s->model.config.sun_dir.y, s->model.config.sun_dir.z};
    diff_create(s, sun, 1, sigma_px, out);
  });
}

int qmcrt_diff_create_suns(qmcrt_scene* s, const float* sun_dirs, int n_suns, float sigma_px, qmcrt_diff** out) {
  return guarded([&] {
    if (!sun_dirs) invalid("sun directions are NULL");
    diff_create(s, sun_dirs, n_suns, sigma_px, out);
  });
}

void qmcrt_diff_free(qmcrt_diff* d) { delete d; }

int qmcrt_diff_set_params(qmcrt_diff* d, const float* aim_offsets, const float* normal_offsets) {
  return guarded([&] {
    diff_checked(d);
    for (int h = 0; h < d->H; ++h) {
      const float2 a = aim_offsets ? make_float2(aim_offsets[2 * h], aim_offsets[2 * h + 1]) : make_float2(0.f, 0.f);
      const float2 n =
          normal_offsets ? make_float2(normal_offsets[2 * h], normal_offsets[2 * h + 1]) : make_float2(0.f, 0.f);
      if (!std::isfinite(a.x) || !std::isfinite(a.y) || !std::isfinite(n.x) || !std::isfinite(n.y))
        invalid("parameters must be finite");
    }
    for (const auto& I : d->batch->inst) {
      for (int h = 0; h < d->H; ++h) {
        qm::PrepItem& it = d->batch->items[I.task_base + h];
        it.aim_offset = aim_offsets ? make_float2(aim_offsets[2 * h], aim_offsets[2 * h + 1]) : make_float2(0.f, 0.f);
        it.normal_offset =
            normal_offsets ? make_float2(normal_offsets[2 * h], normal_offsets[2 * h + 1]) : make_float2(0.f, 0.f);
      }
    }
    d->forward_done = false;
  });
}

int qmcrt_diff_set_target(qmcrt_diff* d, int receiver, const float* target) {
  return guarded([&] {
    diff_checked(d);
    qmcrt_batch* b = d->batch;
    check_receiver(d, receiver);
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
    const size_t bits_bytes = (size_t)std::max<long long>(b->total_chunks, 1) * qm::kChunkIters * sizeof(uint32_t);
    if (d->hit_mode == 0) {
      size_t free_b = 0, total_b = 0;
      cuda_check(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
      d->recompute = bits_bytes > d->d_bits.bytes + free_b / 4;
    } else {
      d->recompute = d->hit_mode == 2;
    }
    if (d->recompute) {
      b->hit_bits = nullptr;  // the adjoint recomputes them
      if (d->d_bits.bytes > (size_t)d->segment_chunks * qm::kChunkIters * sizeof(uint32_t)) d->d_bits.release();
    } else {
      d->d_bits.alloc(bits_bytes);
      b->hit_bits = d->d_bits.as<uint32_t>();
    }
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
    p.light_begin = b->light_begin;
    p.light_end = b->light_end;
    p.grad = d->d_grad.as<double>();
    if (!d->recompute) {
      p.chunk_begin = 0;
      p.total_chunks = b->total_chunks;
      p.hit_bits = d->d_bits.as<uint32_t>();
      cuda_check(qm::launch_diff_backward(p, st), "adjoint kernel");
    } else {
      // Hit records recomputed segment by segment: a hit-bit trace of the
      // segment's chunks (the forward's kernel, mode and rays), then the
      // adjoint over the same chunks.
      const long long seg = std::max<long long>(1, d->segment_chunks);
      d->d_bits.alloc((size_t)std::min(seg, std::max<long long>(b->total_chunks, 1)) * qm::kChunkIters *
                     sizeof(uint32_t));
      b->hit_bits = d->d_bits.as<uint32_t>();
      for (long long c0 = 0; c0 < b->total_chunks; c0 += seg) {
        const long long c1 = std::min(b->total_chunks, c0 + seg);
        cuda_check(batch_launch(b, st, 3, c0, c1), "hit-bit trace");
        p.chunk_begin = c0;
        p.total_chunks = c1;
        p.hit_bits = d->d_bits.as<uint32_t>();
        cuda_check(qm::launch_diff_backward(p, st), "adjoint kernel");
      }
      b->hit_bits = nullptr;
    }
    std::vector<double> slots(d->n_slots * qm::kDiffParams);
    if (!slots.empty())
      cuda_check(cudaMemcpyAsync(slots.data(), d->d_grad.p, slots.size() * sizeof(double), cudaMemcpyDeviceToHost, st),
                 "gradient readback");
    cuda_check(cudaStreamSynchronize(st), "adjoint");
    if (grad) {
      const std::vector<double> g = per_heliostat(d, slots, qm::kDiffParams);
      std::copy(g.begin(), g.end(), grad);
    }
  });
}

int qmcrt_diff_flux(qmcrt_diff* d, int receiver, float* out, int* width, int* height) {
  return guarded([&] {
    diff_checked(d);
    qmcrt_batch* b = d->batch;
    check_receiver(d, receiver);
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

int qmcrt_diff_plain(qmcrt_diff* d, void* stream) {
  return guarded([&] {
    diff_checked(d);
    qmcrt_batch* b = d->batch;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    DeviceGuard guard(b->device);
    // The same parameterised geometry and rays as the forward, binned to
    // the nearest pixel as the plain tracer does.  The forward's hit bits,
    // residual and tangents are untouched, so a pending qmcrt_bwd stays valid.
    batch_prepare(b, st);
    if (b->total_chunks < 0) batch_build_prefix(b);
    cuda_check(cudaMemsetAsync(b->d_images.p, 0, b->d_images.bytes, st), "clear");
    cuda_check(cudaMemsetAsync(b->d_power.p, 0, b->d_power.bytes, st), "clear");
    if (b->light_end > b->light_begin) cuda_check(batch_launch(b, st, 0), "plain trace");
    cuda_check(cudaStreamSynchronize(st), "plain trace");
  });
}

int qmcrt_diff_image(qmcrt_diff* d, int receiver, float* out, int* width, int* height) {
  return guarded([&] {
    diff_checked(d);
    qmcrt_batch* b = d->batch;
    check_receiver(d, receiver);
    const int2 sh = b->image_shape[receiver];
    if (width) *width = sh.x;
    if (height) *height = sh.y;
    if (!out) return;
    DeviceGuard guard(b->device);
    cuda_check(cudaMemcpy(out, b->d_images.as<float>() + b->image_offset[receiver], (size_t)sh.x * sh.y * sizeof(float),
                          cudaMemcpyDeviceToHost),
               "image readback");
  });
}

int qmcrt_diff_power(qmcrt_diff* d, double* per, double* total) {
  return guarded([&] {
    diff_checked(d);
    qmcrt_batch* b = d->batch;
    std::vector<double> slots(d->n_slots);
    DeviceGuard guard(b->device);
    if (!slots.empty())
      cuda_check(cudaMemcpy(slots.data(), b->d_power.p, slots.size() * sizeof(double), cudaMemcpyDeviceToHost),
                 "power readback");
    const std::vector<double> v = per_heliostat(d, slots, 1);
    if (per) std::copy(v.begin(), v.end(), per);
    if (total) {
      // Neumaier-compensated sum of the per-heliostat FP64 powers.
      double sum = 0.0, comp = 0.0;
      for (double x : v) {
        const double t = sum + x;
        comp += std::fabs(sum) >= std::fabs(x) ? (sum - t) + x : (x - t) + sum;
        sum = t;
      }
      *total = sum + comp;
    }
  });
}

int qmcrt_diff_set_hit_records(qmcrt_diff* d, int mode, long long segment_rays) {
  return guarded([&] {
    diff_checked(d);
    if (mode < 0 || mode > 2) invalid("hit-record mode must be 0 (automatic), 1 (checkpoint) or 2 (recompute)");
    if (segment_rays < 0) invalid("segment size must be >= 0 (0 keeps the current one)");
    d->hit_mode = mode;
    if (segment_rays > 0) {
      const long long chunk = trace_chunk_rays();
      d->segment_chunks = std::max<long long>(1, (segment_rays + chunk - 1) / chunk);
    }
    d->forward_done = false;
  });
}

int qmcrt_diff_hit_records(qmcrt_diff* d, int* recomputed, long long* checkpoint_bytes) {
  return guarded([&] {
    diff_checked(d);
    if (recomputed) *recomputed = d->recompute ? 1 : 0;
    if (checkpoint_bytes) *checkpoint_bytes = d->recompute ? 0 : (long long)d->d_bits.bytes;
  });
}

}  // extern "C"
