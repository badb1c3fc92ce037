// Tall-skinny FP64 products and streaming kernels of the Davidson subspace algebra
// (real double or complex double2, column-major).
//   k_sum_parts C = sum over ks of P[ks], fixed order (deterministic)
// and the complex/real arithmetic shared by the tile kernels (gemm_tiles.cuh).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

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

