// mlp.cuh -- the surrogate of the frequency integral of calc_photoion_rate.
//
// For a ray whose emitter spectrum is a normalised blackbody of temperature
// T, and columns M_s [cm^-2] of HI, HeI, HeII, the six integrals
//   I_j(M) = sum_nu w_j(nu) s_nu(T) exp(-sum_s M_s sigma_s(nu)),
//   w_j = sigma_s (j = s) or sigma_s (nu - nu_s)^+ (j = 3 + s),
// are what the reference's 256-bin loop sums (calc_photoion_rate.c:285-387)
// once the photon-conserving cell factor is written as an integral across
// the cell (see photoion_surrogate in photoion.cu).  The network predicts
//   t_j = ln(1 - ln(I_j(M) / I_j(0)))          (t >= 0, range ~[0, 5.5])
// from x = (log10 tau_HI, log10 tau_HeI, log10 tau_HeII, log10 T), with
// tau_s = M_s sigma_s at the species' first absorbing bin; the log-compressed
// target keeps every output O(1) while a thin ray (small ln I/I0) keeps an
// absolute error in ln I equal to that in t.
//
// Architecture: 4 -> 64 -> 64 -> 64 -> 6, SiLU, BF16 weights and activations
// with FP32 accumulation.  The network's input (normalised x) and its last
// hidden layer enter the tensor cores as a BF16 pair hi + lo (an exact
// split of the FP32 value to 16 mantissa bits), so that the two ends that
// set the output's precision are not limited by BF16 rounding; the inner
// activations are single BF16 values.
#pragma once
#include <cuda_bf16.h>

#include "common.cuh"

namespace argot {

constexpr int kMlpIn = 4, kMlpH = 64, kMlpOut = 6;
// parameter layout (FP32 master copy): W1[64][4] b1[64] W2[64][64] b2[64]
// W3[64][64] b3[64] W4[6][64] b4[6]
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kMlpH * kMlpIn;
constexpr int kOffW2 = kOffB1 + kMlpH;
constexpr int kOffB2 = kOffW2 + kMlpH * kMlpH;
constexpr int kOffW3 = kOffB2 + kMlpH;
constexpr int kOffB3 = kOffW3 + kMlpH * kMlpH;
constexpr int kOffW4 = kOffB3 + kMlpH;
constexpr int kOffB4 = kOffW4 + kMlpOut * kMlpH;
constexpr int kMlpParams = kOffB4 + kMlpOut;

// input / output normalisation
constexpr float kTauLo = -6.f, kTauHi = 3.f;     // log10 tau range
constexpr float kTLo = 4.f, kTHi = 5.5f;         // log10 T range
constexpr float kOutShift = 2.75f, kOutScale = 2.75f;

__device__ __forceinline__ float bf16_round(float x) {
  return __bfloat162float(__float2bfloat16_rn(x));
}

// SiLU as the inference kernel evaluates it: z * sigmoid(z) with the
// hardware tanh, sigmoid(z) = (1 + tanh(z/2)) / 2.
__device__ __forceinline__ float tanh_approx(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float silu_fast(float z) {
  const float h = 0.5f * z;
  return fmaf(h, tanh_approx(h), h);
}

}  // namespace argot
