// Tall-skinny FP64 products and streaming kernels of the Davidson subspace algebra
// (real double or complex double2, column-major).
//   k_gemm_tn   P[ks] = A(rows slice ks)^H B(rows slice ks)    (Gram / border blocks)
//   k_sum_parts C = sum over ks of P[ks], fixed order          (deterministic)
//   k_gemm_nn   C (+)= A B, A tall (rows x k), B small (k x n) (rotations, H of a dense matrix)
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

// P[ks][j][i] = sum_{r in slice ks} conj(A[r][i]) B[r][j]; 32 x 32 tile per block.
template <class D>
__global__ void __launch_bounds__(256) k_gemm_tn(const D* __restrict__ A, int64_t lda, const D* __restrict__ B,
                                                 int64_t ldb, D* __restrict__ P, int m, int n, int64_t rows,
                                                 int64_t chunk) {
  __shared__ D As[32][33];
  __shared__ D Bs[32][33];
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32, ks = blockIdx.z;
  const int ti = threadIdx.x & 15, tj = threadIdx.x >> 4;
  D acc[2][2];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) acc[a][b] = Arith<D>::zero();
  const int64_t r0 = ks * chunk, r1 = min(rows, r0 + chunk);
  for (int64_t rb = r0; rb < r1; rb += 32) {
    for (int t = threadIdx.x; t < 1024; t += 256) {
      const int rr = t & 31, q = t >> 5;
      const int64_t r = rb + rr;
      As[rr][q] = (r < r1 && i0 + q < m) ? A[(int64_t)(i0 + q) * lda + r] : Arith<D>::zero();
      Bs[rr][q] = (r < r1 && j0 + q < n) ? B[(int64_t)(j0 + q) * ldb + r] : Arith<D>::zero();
    }
    __syncthreads();
#pragma unroll 8
    for (int rr = 0; rr < 32; ++rr) {
      const D a0 = As[rr][ti], a1 = As[rr][ti + 16];
      const D b0 = Bs[rr][tj], b1 = Bs[rr][tj + 16];
      acc[0][0] = Arith<D>::cmac(acc[0][0], a0, b0);
      acc[1][0] = Arith<D>::cmac(acc[1][0], a1, b0);
      acc[0][1] = Arith<D>::cmac(acc[0][1], a0, b1);
      acc[1][1] = Arith<D>::cmac(acc[1][1], a1, b1);
    }
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const int i = i0 + ti + 16 * a, j = j0 + tj + 16 * b;
      if (i < m && j < n) P[((int64_t)ks * n + j) * m + i] = acc[a][b];
    }
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

// C[r][j] (+)= sum_p A[r][p] B[p][j]; tile 64 rows x 32 columns.
template <class D>
__global__ void __launch_bounds__(256) k_gemm_nn(const D* __restrict__ A, int64_t lda, const D* __restrict__ B,
                                                 int64_t ldb, D* __restrict__ C, int64_t ldc, int64_t rows, int n,
                                                 int k, int accumulate) {
  __shared__ D As[16][64];
  __shared__ D Bs[16][33];
  const int64_t r0 = (int64_t)blockIdx.x * 64;
  const int j0 = blockIdx.y * 32;
  const int tr = threadIdx.x & 31, tc = threadIdx.x >> 5;
  D acc[2][4];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = Arith<D>::zero();
  for (int pb = 0; pb < k; pb += 16) {
    for (int t = threadIdx.x; t < 16 * 64; t += 256) {
      const int rr = t & 63, q = t >> 6;
      const int p = pb + q;
      const int64_t r = r0 + rr;
      As[q][rr] = (p < k && r < rows) ? A[(int64_t)p * lda + r] : Arith<D>::zero();
    }
    for (int t = threadIdx.x; t < 16 * 32; t += 256) {
      const int q = t & 15, cc = t >> 4;
      const int p = pb + q, j = j0 + cc;
      Bs[q][cc] = (p < k && j < n) ? B[(int64_t)j * ldb + p] : Arith<D>::zero();
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const D a0 = As[q][tr], a1 = As[q][tr + 32];
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const D bb = Bs[q][tc + 8 * b];
        acc[0][b] = Arith<D>::mac(acc[0][b], a0, bb);
        acc[1][b] = Arith<D>::mac(acc[1][b], a1, bb);
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int64_t r = r0 + tr + 32 * a;
      const int j = j0 + tc + 8 * b;
      if (r < rows && j < n) {
        D& out = C[(int64_t)j * ldc + r];
        out = accumulate ? Arith<D>::add(out, acc[a][b]) : acc[a][b];
      }
    }
}

}  // namespace bg
