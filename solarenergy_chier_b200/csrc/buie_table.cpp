// Host half of the reference's Buie sun-shape sampler: kappa, gamma and the
// trapezoidal CDF of the core intensity (Scene/SceneProcessor.cu:7-44 and
// :204-239).  Float arithmetic in the reference's order, -ffp-contract=off.
#include <cmath>

#include "pools.h"

namespace qm {

namespace {
// samplelights::sunshape_intensity (Scene/SceneProcessor.cu:7-10).
float core_intensity(float theta) { return cosf(0.326f * theta) / cosf(0.308f * theta); }
// samplelights::integration_larger_than_465_intensity (Scene/SceneProcessor.cu:12-15).
float tail_integral(float theta, float k, float gamma) { return expf(k) / (gamma + 1) * powf(theta, gamma + 1); }
}  // namespace

BuieHost build_buie_table(float csr, int num_group) {
  BuieHost t;
  const float upper_lm = 4.65f;
  const float k = 0.9f * logf(13.5f * csr) * powf(csr, -0.3f);
  const float gamma = 2.2f * logf(0.52f * csr) * powf(csr, 0.43f) - 0.1f;
  const float i_465_930 = tail_integral(9.3f, k, gamma) - tail_integral(upper_lm, k, gamma);
  t.cdf.assign(num_group + 1, make_float2(0.f, 0.f));
  t.k.assign(num_group, 0.f);
  const float length_interval = upper_lm / float(num_group);
  float x = 0.0f;
  float hist_pre = core_intensity(x);
  for (int i = 1; i <= num_group; ++i) {
    x += length_interval;
    float hist_cur = core_intensity(x);
    float subarea = (hist_cur + hist_pre) / 2.0f * length_interval;
    t.cdf[i].x = x;
    t.cdf[i].y = subarea + t.cdf[i - 1].y;
    t.k[i - 1] = length_interval / subarea;
    hist_pre = hist_cur;
  }
  t.less_465 = t.cdf[num_group].y;
  t.kappa = k;
  t.gamma = gamma;
  t.A = t.less_465 + i_465_930;
  t.B = (gamma + 1) / expf(k);
  t.C = powf(upper_lm, gamma + 1);
  return t;
}

}  // namespace qm
