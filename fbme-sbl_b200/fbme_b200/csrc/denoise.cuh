// The UAMP Gaussian denoiser of one coefficient, shared by the elementwise
// denoiser (uamp.cu) and the FFT stage that fuses it into its epilogue
// (fft.cu).
#pragma once

#include <stdint.h>

#include "common.cuh"
#include "stage.cuh"

namespace fbme {

// Gaussian denoiser with damping and the fused ARD prior update
// (triton_kernels.py:140-192; solver.py:2832-2850, 1600-1607).
struct DenoiseArgs {
  float2* mu;
  float* var;
  float* gamma;
  const float* pv;
  const float* floor_;
  double* part;
  uint32_t* keys;  // optional: score key of |mu|^2 + v for the top-K
  float damping, prior_damping, prior_max, hyper_shape, hyper_rate;
  float inv_hyper;  // 1 / (1 + hyper_shape)
  int update_prior;
};

FBME_DEV uint32_t float_key(float f) {
  const uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

// One coefficient of the denoiser (triton_kernels.py:140-184): new mean,
// variance, relevance and (optionally) prior variance.  Divisions use the
// fast reciprocal path (<= 2 ulp), as the fused Triton kernel's `/` does.
struct DenoiseOut {
  float2 mean;
  float variance, rel, gamma;
};

FBME_DEV DenoiseOut denoise_math(const DenoiseArgs& a, float prior, float2 om, float ov_raw,
                                 float2 L, float pv, float fl) {
  DenoiseOut o;
  const float ov = fmaxf(ov_raw, kTiny);
  const float den = fmaxf(prior + pv, kTiny);
  const float gain = __fdividef(prior, den);
  const float2 pm = make_float2(om.x + pv * L.x, om.y + pv * L.y);
  const float keep = a.damping, upd = 1.0f - a.damping;
  o.mean = make_float2(keep * om.x + upd * (gain * pm.x), keep * om.y + upd * (gain * pm.y));
  const float cv = __fdividef(prior * pv, den);
  o.variance = fmaxf(keep * ov + upd * cv, kTiny);
  o.rel = fmaxf(0.0f, fminf(1.0f, 1.0f - __fdividef(o.variance, fmaxf(prior, kTiny))));
  const float second = o.mean.x * o.mean.x + o.mean.y * o.mean.y + o.variance;
  float cand = (second + a.hyper_rate) * a.inv_hyper;
  cand = fmaxf(fl, fminf(a.prior_max, cand));
  o.gamma = fmaxf(a.prior_damping * prior + (1.0f - a.prior_damping) * cand, fl);
  return o;
}

}  // namespace fbme
