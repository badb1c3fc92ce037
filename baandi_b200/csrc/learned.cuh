// Learned preconditioner: a per-G-vector MLP 5 -> 64 -> 64 -> 1 (GELU) whose output is a
// log-multiplier on the TPA factor,
//   c_g = -tpa(t_g, s_j) exp(clamp(m(f_gj), -kClamp, kClamp)) r_g,
// with r = H x_j - lambda_j x_j, t_g the kinetic diagonal, s_j the band's kinetic scale
// (the TPA scale, max(0.1, sum |x|^2 t / sum |x|^2)) and the five inputs
//   f0 = log(max(t_g / s_j, 1e-4))          the TPA ratio
//   f1 = log(t_g + 0.05)                    |k+G|^2 / 2
//   f2 = log(s_j)                           band kinetic energy
//   f3 = lambda_j                           Ritz value (Ha)
//   f4 = log(clamp(|r_g| / rms_j(r), 1e-6, 1e6))   local residual magnitude.
// Weights are BF16 (round to nearest even); the layers accumulate in FP32.  A network
// whose last layer is zero is exactly TPA (exp(0) = 1).
#pragma once
#include <cuda_bf16.h>
#include <cstdint>

namespace bg {
namespace learned {

constexpr int kIn = 5, kHid = 64;
// Parameter layout (one array): W1 [64][5], b1 [64], W2 [64][64] (row = output),
// b2 [64], w3 [64], b3.
constexpr int oW1 = 0;
constexpr int oB1 = oW1 + kHid * kIn;
constexpr int oW2 = oB1 + kHid;
constexpr int oB2 = oW2 + kHid * kHid;
constexpr int oW3 = oB2 + kHid;
constexpr int oB3 = oW3 + kHid;
constexpr int kParams = oB3 + 1;  // 4609
constexpr float kClamp = 3.0f;

// GELU, tanh form: 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))), and its derivative.
__device__ __forceinline__ float gelu(float x) {
  const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
  return 0.5f * x * (1.0f + tanhf(u));
}
__device__ __forceinline__ float gelu_grad(float x) {
  const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
  const float th = tanhf(u);
  const float du = 0.7978845608028654f * (1.0f + 3.0f * 0.044715f * x * x);
  return 0.5f * (1.0f + th) + 0.5f * x * (1.0f - th * th) * du;
}

__device__ __forceinline__ void features(double t, double s, double lam, double rho, float* f) {
  f[0] = (float)log(fmax(t / s, 1e-4));
  f[1] = (float)log(t + 0.05);
  f[2] = (float)log(s);
  f[3] = (float)lam;
  f[4] = (float)log(fmin(fmax(rho, 1e-6), 1e6));
}

// Network output m(f) with the parameters as floats in shared memory (w).
__device__ __forceinline__ float forward(const float* __restrict__ w, const float* f) {
  float h1[kHid];
#pragma unroll
  for (int i = 0; i < kHid; ++i) {
    float a = w[oB1 + i];
#pragma unroll
    for (int k = 0; k < kIn; ++k) a = fmaf(w[oW1 + i * kIn + k], f[k], a);
    h1[i] = gelu(a);
  }
  float out = w[oB3];
#pragma unroll 4
  for (int o = 0; o < kHid; ++o) {
    float a = w[oB2 + o];
#pragma unroll
    for (int i = 0; i < kHid; ++i) a = fmaf(w[oW2 + o * kHid + i], h1[i], a);
    out = fmaf(w[oW3 + o], gelu(a), out);
  }
  return out;
}

// Multiplier on the TPA factor from the network output.
__device__ __forceinline__ double multiplier(float m) { return (double)expf(fminf(fmaxf(m, -kClamp), kClamp)); }

// BF16 parameters (global) -> floats in shared memory; the whole block takes part and
// meets at a barrier.
__device__ __forceinline__ void load_params(const __nv_bfloat16* __restrict__ p, float* w) {
  for (int i = threadIdx.x; i < kParams; i += blockDim.x) w[i] = __bfloat162float(p[i]);
  __syncthreads();
}

}  // namespace learned
}  // namespace bg
