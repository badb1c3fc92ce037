// Tall-skinny FP64 products and streaming kernels of the Davidson subspace algebra
// (real double or complex double2, column-major).
//   k_sum_parts C = sum over ks of P[ks], fixed order (deterministic)
// and the complex/real arithmetic shared by the tile kernels (gemm_tiles.cuh).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include "learned.cuh"

namespace bg {

template <class D>
struct Arith;
template <>
struct Arith<double> {
  __device__ static double zero() { return 0.0; }
  __device__ static double cmac(double acc, double a, double b) { return fma(a, b, acc); }  // conj(a) b
  __device__ static double mac(double acc, double a, double b) { return fma(a, b, acc); }
  __device__ static double add(double a, double b) { return a + b; }
  __device__ static double scale(double s, double a) { return s * a; }
  __device__ static double norm2(double a) { return a * a; }
};
template <>
struct Arith<double2> {
  __device__ static double2 zero() { return make_double2(0.0, 0.0); }
  __device__ static double2 cmac(double2 acc, double2 a, double2 b) {
    acc.x = fma(a.x, b.x, fma(a.y, b.y, acc.x));
    acc.y = fma(a.x, b.y, fma(-a.y, b.x, acc.y));
    return acc;
  }
  __device__ static double2 mac(double2 acc, double2 a, double2 b) {
    acc.x = fma(a.x, b.x, fma(-a.y, b.y, acc.x));
    acc.y = fma(a.x, b.y, fma(a.y, b.x, acc.y));
    return acc;
  }
  __device__ static double2 add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
  __device__ static double2 scale(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
  __device__ static double norm2(double2 a) { return a.x * a.x + a.y * a.y; }
};

// Positive TPA damping of kinetic coordinate t at band scale s (crates/dft-solvers/src/
// lib.rs:194-206; the reciprocal form for t > s avoids polynomial overflow).
__device__ __forceinline__ double tpa_weight(double t, double s) {
  const double x = t / s;
  if (x <= 1.0) {
    const double p = 27.0 + x * (18.0 + x * (12.0 + x * 8.0));
    return p / (p + 16.0 * x * x * x * x);
  }
  const double y = s / t;
  const double p = y * (8.0 + y * (12.0 + y * (18.0 + y * 27.0)));
  return p / (p + 16.0);
}

// Reference Davidson smooth denominator (crates/dft-solvers/src/ref_davidson.rs:418-422).
__device__ __forceinline__ double smooth_denominator(double h, double e) {
  const double x = 2.0 * (h - e);
  const double z = fabs(x - 1.0);
  return 0.25 * (2.0 * fmax(x, 1.0) + 1.0 / (sqrt(1.0 + z * z) + z));
}

// Block-wide sum (blockDim.x = 256) through a shared array of 256 doubles.
__device__ __forceinline__ double block_sum256(double v, double* red) {
  red[threadIdx.x] = v;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  const double r = red[0];
  __syncthreads();
  return r;
}

// Correction of one band column from its Ritz vector x and H x (rows entries):
// kind 0 (smooth) out = (hx - e x) / d(diag, e); kind 1 (TPA) out = -(hx - e x)
// tpa(diag, s) with s = max(0.1, sum |x|^2 diag / sum |x|^2), diag = kinetic;
// kind 2 (Ritz shift) out = -(hx - e x) / max(diag - e, 0.1); kind 3 (learned) the TPA
// factor times exp(clamp(m(f))) of the per-G network whose parameters `net` holds as
// floats in shared memory (learned.cuh).  Returns |out|^2 (all threads of the 256-thread
// block); res2, when given, receives the raw residual's |HX_j - lambda_j X_j|^2.
template <class D, bool LEARNED = false>
__device__ double correction_column(const D* __restrict__ x, const D* __restrict__ hx,
                                    const double* __restrict__ diag, double e, int kind, int64_t rows,
                                    D* __restrict__ out, double* red, const float* net = nullptr,
                                    double* res2 = nullptr) {
  if constexpr (LEARNED) kind = 3;
  double scale = 0.0, rms = 0.0;
  if (kind == 1 || kind == 3) {
    double w = 0.0, wt = 0.0;
    for (int64_t r = threadIdx.x; r < rows; r += blockDim.x) {
      const double a = Arith<D>::norm2(x[r]);
      w += a;
      wt += a * diag[r];
    }
    w = block_sum256(w, red);
    wt = block_sum256(wt, red);
    scale = fmax(wt / w, 0.1);
  }
  if (LEARNED) {
    double q = 0.0;
    for (int64_t r = threadIdx.x; r < rows; r += blockDim.x)
      q += Arith<D>::norm2(Arith<D>::add(hx[r], Arith<D>::scale(-e, x[r])));
    rms = sqrt(block_sum256(q, red) / (double)rows);
  }
  double acc = 0.0, racc = 0.0;
  for (int64_t r = threadIdx.x; r < rows; r += blockDim.x) {
    const D res = Arith<D>::add(hx[r], Arith<D>::scale(-e, x[r]));
    if (res2) racc += Arith<D>::norm2(res);
    double f;
    if (kind == 1)
      f = -tpa_weight(diag[r], scale);
    else if (LEARNED) {
      float in[learned::kIn];
      learned::features(diag[r], scale, e, rms > 0.0 ? sqrt(Arith<D>::norm2(res)) / rms : 1.0, in);
      f = -tpa_weight(diag[r], scale) * learned::multiplier(learned::forward(net, in));
    }
    else if (kind == 2)
      f = -1.0 / fmax(diag[r] - e, 0.1);
    else
      f = 1.0 / smooth_denominator(diag[r], e);
    const D v = Arith<D>::scale(f, res);
    out[r] = v;
    acc += Arith<D>::norm2(v);
  }
  if (res2) *res2 = block_sum256(racc, red);   // |HX_j - lambda_j X_j|^2 (every thread)
  return block_sum256(acc, red);
}

template <class D>
__global__ void k_sum_parts(const D* __restrict__ P, int ks, int m, int n, D* __restrict__ C, int64_t ldc) {
  const int64_t total = (int64_t)m * n;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = t / m, i = t - j * m;
    D s = Arith<D>::zero();
    for (int k = 0; k < ks; ++k) s = Arith<D>::add(s, P[(int64_t)k * total + t]);
    C[j * ldc + i] = s;
  }
}

}  // namespace bg

