// warmnet.cuh -- the learned warm start: a per-particle MLP
// 12 -> 64 -> 64 -> 2 with GELU, BF16 operands and FP32 accumulation on the
// tensor cores (tcgen05, accumulators in TMEM).  No reference counterpart:
// it replaces the previous-step warm starts of the DFSPH solves
// (warm_start_divergence_solve_0, runner.hpp:3230-3249, and
// warm_start_pressure_solve0, runner.hpp:3430-3449) by a prediction of the
// converged kappa_v and kappa; the solves' own tolerances still decide how
// many iterations run.
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"
#include "engine.hpp"

namespace alb {

constexpr int kWarmIn = AL_WARM_NUM_FEATURES;  // 12
constexpr int kWarmInPad = 16;                  // K of the first MMA
constexpr int kWarmHidden = AL_WARM_HIDDEN;     // 64
constexpr int kWarmOut = AL_WARM_NUM_OUTPUTS;   // 2
constexpr int kWarmOutPad = 16;                 // N of the last MMA
// offsets into the flat FP32 parameter array
constexpr int kOffW1 = 0;                                  // W1[64][12]
constexpr int kOffB1 = kOffW1 + kWarmHidden * kWarmIn;     // b1[64]
constexpr int kOffW2 = kOffB1 + kWarmHidden;               // W2[64][64]
constexpr int kOffB2 = kOffW2 + kWarmHidden * kWarmHidden; // b2[64]
constexpr int kOffW3 = kOffB2 + kWarmHidden;               // W3[2][64]
constexpr int kOffB3 = kOffW3 + kWarmOut * kWarmHidden;    // b3[2]
static_assert(kOffB3 + kWarmOut == AL_WARM_NUM_PARAMS, "parameter layout");

// Kernel-side copy of al_warm_net.
struct WarmNetDev {
  const float* params;
  float shift[kWarmIn];
  float scale[kWarmIn];
  float out_scale[kWarmOut];
};

inline WarmNetDev to_warm_dev(const al_warm_net& n) {
  WarmNetDev d;
  d.params = n.params;
  for (int k = 0; k < kWarmIn; ++k) {
    d.shift[k] = n.feature_shift[k];
    d.scale[k] = n.feature_scale[k];
  }
  for (int k = 0; k < kWarmOut; ++k) d.out_scale[k] = n.output_scale[k];
  return d;
}

// GELU in the tanh form of Hendrycks & Gimpel (2016):
// g(x) = x/2 (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))), with the hardware
// tanh approximation; g' for the backward pass.
__device__ __forceinline__ float tanh_hw(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
constexpr float kGeluC = 0.7978845608028654f;  // sqrt(2 / pi)
constexpr float kGeluA = 0.044715f;
__device__ __forceinline__ float gelu(float x) {
  const float t = tanh_hw(kGeluC * (x + kGeluA * x * x * x));
  return 0.5f * x * (1.0f + t);
}
__device__ __forceinline__ float gelu_grad(float x) {
  const float t = tanh_hw(kGeluC * (x + kGeluA * x * x * x));
  return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * kGeluC * (1.0f + 3.0f * kGeluA * x * x);
}

// Normalised features of one particle: (x - shift) * scale.
__device__ __forceinline__ void warm_normalize(const WarmNetDev& net, const float* raw,
                                               float (&xn)[kWarmInPad]) {
#pragma unroll
  for (int k = 0; k < kWarmIn; ++k) xn[k] = (raw[k] - net.shift[k]) * net.scale[k];
#pragma unroll
  for (int k = kWarmIn; k < kWarmInPad; ++k) xn[k] = 0.f;
}

// out[p][0..1] = net(features[p]) * out_scale for p < n (features: raw
// [n][12] FP32).  Raises err[0] if a tensor-core wait timed out.  With
// `skip` (device word) nonzero when the kernel runs, it returns at once.
int warm_forward(al_engine* e, const WarmNetDev& net, const float* features, uint32_t n,
                 float* out, uint32_t* err, cudaStream_t st, const uint32_t* skip = nullptr);

}  // namespace alb
