// FP64 tall-skinny products on the CUDA cores (real double or complex double2), with
// shared-memory tiles filled by cp.async one step ahead of the arithmetic and a 4 x 4
// register tile per thread.  FP64 on sm_100a runs at the same rate on the CUDA cores as
// through DMMA, and tcgen05 has no FP64 kind.
//   tn_tile: P = A[r0:r1, :]^H B[r0:r1, :] for one 32 x 32 output tile (split over rows)
//   nn_tile: C (+)= A B for one 64-row x 32-column output tile, A tall, B small
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "blas_dev.cuh"

namespace bg {
namespace tiles {

constexpr int kBK = 16;  // rows (TN) or inner indices (NN) per shared-memory step

template <class D>
__device__ __forceinline__ void async_copy(D* dst, const D* src) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  if constexpr (sizeof(D) == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src));
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src));
}
__device__ __forceinline__ void async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// 64 threads; thread (ti, tj) owns outputs i = 8a + ti, j = 8b + tj of the 32 x 32 tile
// (interleaved so that the lanes of a warp read consecutive shared-memory words).
// A: rows x m (column-major, lda), B: rows x n (ldb); output written to
// P[j * ldp + i] for the valid i < m, j < n (relative to the tile origin i0, j0).
template <class D>
__device__ __forceinline__ void tn_tile(const D* __restrict__ A, int64_t lda, const D* __restrict__ B,
                                        int64_t ldb, int i0, int j0, int m, int n, int64_t r0, int64_t r1,
                                        D* __restrict__ P, int64_t ldp) {
  __shared__ __align__(16) D As[2][kBK][32];
  __shared__ __align__(16) D Bs[2][kBK][32];
  const int tid = threadIdx.x;
  const int ti = tid & 7, tj = tid >> 3;
  D acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = Arith<D>::zero();
  // one step loads kBK x 32 values of A and of B: 512 each, 8 per thread
  auto load = [&](int buf, int64_t rb) {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int e = tid + 64 * q;
      const int rr = e & (kBK - 1), c = e >> 4;  // 16 rows x 32 columns
      const int64_t r = rb + rr;
      const bool rok = r < r1;
      D* da = &As[buf][rr][c];
      D* db = &Bs[buf][rr][c];
      if (rok && i0 + c < m)
        async_copy(da, A + (int64_t)(i0 + c) * lda + r);
      else
        *da = Arith<D>::zero();
      if (rok && j0 + c < n)
        async_copy(db, B + (int64_t)(j0 + c) * ldb + r);
      else
        *db = Arith<D>::zero();
    }
    async_commit();
  };
  const int64_t steps = (r1 - r0 + kBK - 1) / kBK;
  if (steps > 0) load(0, r0);
  for (int64_t s = 0; s < steps; ++s) {
    const int cur = s & 1;
    if (s + 1 < steps) {
      load(cur ^ 1, r0 + (s + 1) * kBK);
      async_wait<1>();
    } else {
      async_wait<0>();
    }
    __syncthreads();
#pragma unroll
    for (int rr = 0; rr < kBK; ++rr) {
      D a[4], b[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        a[q] = As[cur][rr][q * 8 + ti];
        b[q] = Bs[cur][rr][q * 8 + tj];
      }
#pragma unroll
      for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int y = 0; y < 4; ++y) acc[x][y] = Arith<D>::cmac(acc[x][y], a[x], b[y]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int x = 0; x < 4; ++x)
#pragma unroll
    for (int y = 0; y < 4; ++y) {
      const int i = i0 + x * 8 + ti, j = j0 + y * 8 + tj;
      if (i < m && j < n) P[(int64_t)j * ldp + i] = acc[x][y];
    }
}

// 48 x 48 tiles of P = A^H B for the Davidson's Grams (m, n <= the basis capacity, 48 for
// the k-point cells): 256 threads; thread (ti, tj) = (lane mod 16, 2 warp + lane / 16)
// owns outputs i = i0 + ti + 16 a, j = j0 + 3 tj + b (a, b < 3).  A warp's columns are
// uniform, so a warp whose columns all lie at or beyond n skips the arithmetic.  The rows
// stream through kStages48 shared-memory stages of kBK48 rows each, filled by cp.async
// kStages48 - 1 stages ahead of the arithmetic; a stage holds each column's kBK48 rows
// contiguously with a pitch of kBK48 + 1 elements, so both the fill (consecutive threads,
// consecutive rows) and the arithmetic's reads (16 columns of one row per half-warp, 17
// elements apart) meet no bank conflicts.  Dynamic shared memory: tn48_smem_bytes<D>().
constexpr int kBK48 = 16;
constexpr int kStages48 = 4;
constexpr int kPitch48 = kBK48 + 1;
template <class D>
constexpr size_t tn48_smem_bytes() {
  return (size_t)2 * kStages48 * 48 * kPitch48 * sizeof(D);
}
template <class D>
__device__ __forceinline__ void tn_tile48(const D* __restrict__ A, int64_t lda, const D* __restrict__ B,
                                          int64_t ldb, int i0, int j0, int m, int n, int64_t r0, int64_t r1,
                                          D* __restrict__ P, int64_t ldp) {
  extern __shared__ __align__(16) unsigned char tn48_smem[];
  D* As = reinterpret_cast<D*>(tn48_smem);  // [stage][48 columns][kPitch48 rows]
  D* Bs = As + kStages48 * 48 * kPitch48;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int ti = lane & 15, tj = 2 * warp + (lane >> 4);
  const bool warp_live = j0 + 6 * warp < n;
  D acc[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) acc[a][b] = Arith<D>::zero();
  // one stage: kBK48 rows x 48 columns of A and of B, 6 elements per thread
  auto load = [&](int buf, int64_t rb) {
    for (int e = tid; e < 2 * 48 * kBK48; e += 256) {
      const int mat = e / (48 * kBK48), idx = e - mat * (48 * kBK48);
      const int rr = idx % kBK48, c = idx / kBK48;
      const int64_t r = rb + rr;
      D* dst = (mat == 0 ? As : Bs) + (buf * 48 + c) * kPitch48 + rr;
      const bool ok = r < r1 && (mat == 0 ? i0 + c < m : j0 + c < n);
      if (ok)
        async_copy(dst, mat == 0 ? A + (int64_t)(i0 + c) * lda + r : B + (int64_t)(j0 + c) * ldb + r);
      else
        *dst = Arith<D>::zero();
    }
    async_commit();
  };
  const int64_t steps = (r1 - r0 + kBK48 - 1) / kBK48;
  // one cp.async group per stage, empty ones past the end, so that waiting for all but
  // the newest kStages48 - 2 groups always means the current stage has landed
#pragma unroll
  for (int s = 0; s < kStages48 - 1; ++s) {
    if (s < steps)
      load(s, r0 + s * kBK48);
    else
      async_commit();
  }
  for (int64_t s = 0; s < steps; ++s) {
    async_wait<kStages48 - 2>();
    __syncthreads();  // stage s visible to all; every thread is done with stage s - 1
    const int64_t nxt = s + kStages48 - 1;
    if (nxt < steps)
      load((int)(nxt % kStages48), r0 + nxt * kBK48);  // refills the buffer of stage s - 1
    else
      async_commit();
    if (warp_live) {
      const D* as = As + (int)(s % kStages48) * 48 * kPitch48;
      const D* bs = Bs + (int)(s % kStages48) * 48 * kPitch48;
#pragma unroll
      for (int rr = 0; rr < kBK48; ++rr) {
        D a[3], b[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          a[q] = as[(ti + 16 * q) * kPitch48 + rr];
          b[q] = bs[(3 * tj + q) * kPitch48 + rr];
        }
#pragma unroll
        for (int x = 0; x < 3; ++x)
#pragma unroll
          for (int y = 0; y < 3; ++y) acc[x][y] = Arith<D>::cmac(acc[x][y], a[x], b[y]);
      }
    }
  }
  async_wait<0>();
#pragma unroll
  for (int x = 0; x < 3; ++x)
#pragma unroll
    for (int y = 0; y < 3; ++y) {
      const int i = i0 + ti + 16 * x, j = j0 + 3 * tj + y;
      if (i < m && j < n) P[(int64_t)j * ldp + i] = acc[x][y];
    }
}

// 128 threads; thread (tr, tc) owns rows r0 + 16a + tr and columns j0 + 8b + tc of a
// 64 x 32 tile of C (rows x n, ldc); A: rows x k (lda), B: k x n (ldb).
template <class D, bool SKIP_EMPTY = false>
__device__ __forceinline__ void nn_tile(const D* __restrict__ A, int64_t lda, const D* __restrict__ B,
                                        int64_t ldb, D* __restrict__ C, int64_t ldc, int64_t rows, int n, int k,
                                        int64_t r0, int j0, bool accumulate) {
  __shared__ __align__(16) D As[2][kBK][64];
  __shared__ __align__(16) D Bs[2][kBK][32];
  const int tid = threadIdx.x;
  const int tr = tid & 15, tc = tid >> 4;
  D acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = Arith<D>::zero();
  auto load = [&](int buf, int pb) {
#pragma unroll
    for (int q = 0; q < 8; ++q) {  // A: kBK x 64
      const int e = tid + 128 * q;
      const int rr = e & 63, p = e >> 6;
      const int64_t r = r0 + rr;
      D* d = &As[buf][p][rr];
      if (r < rows && pb + p < k)
        async_copy(d, A + (int64_t)(pb + p) * lda + r);
      else
        *d = Arith<D>::zero();
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {  // B: kBK x 32
      const int e = tid + 128 * q;
      const int p = e & (kBK - 1), c = e >> 4;
      D* d = &Bs[buf][p][c];
      if (pb + p < k && j0 + c < n)
        async_copy(d, B + (int64_t)(j0 + c) * ldb + pb + p);
      else
        *d = Arith<D>::zero();
    }
    async_commit();
  };
  // SKIP_EMPTY: the 8-column groups of the tile beyond n (the same for every thread) skip
  // their multiply-adds (pays where n is often below the tile width, the Davidson's
  // rotations of n <= bands columns)
  const int ny = SKIP_EMPTY ? min(4, (n - j0 + 7) / 8) : 4;
  const int steps = (k + kBK - 1) / kBK;
  if (steps > 0) load(0, 0);
  for (int s = 0; s < steps; ++s) {
    const int cur = s & 1;
    if (s + 1 < steps) {
      load(cur ^ 1, (s + 1) * kBK);
      async_wait<1>();
    } else {
      async_wait<0>();
    }
    __syncthreads();
#pragma unroll
    for (int p = 0; p < kBK; ++p) {
      D a[4], b[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        a[q] = As[cur][p][q * 16 + tr];
        b[q] = Bs[cur][p][q * 8 + tc];
      }
#pragma unroll
      for (int y = 0; y < 4; ++y)
        if (y < ny) {
#pragma unroll
          for (int x = 0; x < 4; ++x) acc[x][y] = Arith<D>::mac(acc[x][y], a[x], b[y]);
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int x = 0; x < 4; ++x)
#pragma unroll
    for (int y = 0; y < 4; ++y) {
      const int64_t r = r0 + x * 16 + tr;
      const int j = j0 + y * 8 + tc;
      if (r < rows && j < n) {
        D& out = C[(int64_t)j * ldc + r];
        out = accumulate ? Arith<D>::add(out, acc[x][y]) : acc[x][y];
      }
    }
}

// 64 x 64 tiles of C (+)= A B, A tall (rows x k, column-major), B small (k x n): 256
// threads; thread (tr, tc) = (tid mod 16, tid / 16) owns rows r0 + tr + 16 x and columns
// j0 + tc + 16 y (x, y < 4).  The inner index streams through kStages64 shared-memory
// stages of kBK rows of A (64 rows each, contiguous as in memory) and kBK entries of each
// of 64 columns of B (a column's entries contiguous, pitch kBK + 1), filled by cp.async
// kStages64 - 1 stages ahead; neither the fill nor the arithmetic's reads meet bank
// conflicts.  SKIP_EMPTY skips the 16-column groups at or beyond n.  Dynamic shared
// memory: nn64_smem_bytes<D>().
constexpr int kStages64 = 3;
constexpr int kPitchB64 = kBK + 1;
template <class D>
constexpr size_t nn64_smem_bytes() {
  return (size_t)kStages64 * (kBK * 64 + 64 * kPitchB64) * sizeof(D);
}
template <class D, bool SKIP_EMPTY = false>
__device__ __forceinline__ void nn_tile64(const D* __restrict__ A, int64_t lda, const D* __restrict__ B,
                                          int64_t ldb, D* __restrict__ C, int64_t ldc, int64_t rows, int n, int k,
                                          int64_t r0, int j0, bool accumulate) {
  extern __shared__ __align__(16) unsigned char nn64_smem[];
  D* As = reinterpret_cast<D*>(nn64_smem);     // [stage][kBK][64 rows]
  D* Bs = As + kStages64 * kBK * 64;           // [stage][64 columns][kPitchB64]
  const int tid = threadIdx.x;
  const int tr = tid & 15, tc = tid >> 4;
  D acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = Arith<D>::zero();
  auto load = [&](int buf, int pb) {
    D* as = As + buf * kBK * 64;
    D* bs = Bs + buf * 64 * kPitchB64;
#pragma unroll
    for (int q = 0; q < 4; ++q) {  // A: kBK x 64, consecutive threads on consecutive rows
      const int e = tid + 256 * q;
      const int rr = e & 63, p = e >> 6;
      const int64_t r = r0 + rr;
      D* d = as + p * 64 + rr;
      if (r < rows && pb + p < k)
        async_copy(d, A + (int64_t)(pb + p) * lda + r);
      else
        *d = Arith<D>::zero();
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {  // B: 64 columns x kBK, consecutive threads on consecutive entries
      const int e = tid + 256 * q;
      const int p = e & (kBK - 1), c = e >> 4;
      D* d = bs + c * kPitchB64 + p;
      if (pb + p < k && j0 + c < n)
        async_copy(d, B + (int64_t)(j0 + c) * ldb + pb + p);
      else
        *d = Arith<D>::zero();
    }
    async_commit();
  };
  const int ny = SKIP_EMPTY ? min(4, max(0, (n - j0 - tc + 15) / 16)) : 4;
  const int steps = (k + kBK - 1) / kBK;
#pragma unroll
  for (int s = 0; s < kStages64 - 1; ++s) {
    if (s < steps)
      load(s, s * kBK);
    else
      async_commit();
  }
  for (int s = 0; s < steps; ++s) {
    async_wait<kStages64 - 2>();
    __syncthreads();  // stage s visible to all; every thread is done with stage s - 1
    const int nxt = s + kStages64 - 1;
    if (nxt < steps)
      load(nxt % kStages64, nxt * kBK);  // refills the buffer of stage s - 1
    else
      async_commit();
    const D* as = As + (s % kStages64) * kBK * 64;
    const D* bs = Bs + (s % kStages64) * 64 * kPitchB64;
#pragma unroll
    for (int p = 0; p < kBK; ++p) {
      D a[4], b[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        a[q] = as[p * 64 + q * 16 + tr];
        b[q] = bs[(q * 16 + tc) * kPitchB64 + p];
      }
#pragma unroll
      for (int y = 0; y < 4; ++y)
        if (y < ny) {
#pragma unroll
          for (int x = 0; x < 4; ++x) acc[x][y] = Arith<D>::mac(acc[x][y], a[x], b[y]);
        }
    }
  }
  async_wait<0>();
#pragma unroll
  for (int x = 0; x < 4; ++x)
#pragma unroll
    for (int y = 0; y < 4; ++y) {
      const int64_t r = r0 + x * 16 + tr;
      const int j = j0 + y * 16 + tc;
      if (r < rows && j < n) {
        D& out = C[(int64_t)j * ldc + r];
        out = accumulate ? Arith<D>::add(out, acc[x][y]) : acc[x][y];
      }
    }
}

}  // namespace tiles
}  // namespace bg

namespace bg {
// P[ks][j][i] = sum_{r in slice ks} conj(A[r][i]) B[r][j]; one 32 x 32 tile per block (64 threads).
template <class D>
__global__ void __launch_bounds__(64) k_gemm_tn(const D* __restrict__ A, int64_t lda, const D* __restrict__ B,
                                                int64_t ldb, D* __restrict__ P, int m, int n, int64_t rows,
                                                int64_t chunk) {
  const int64_t r0 = (int64_t)blockIdx.z * chunk, r1 = min(rows, r0 + chunk);
  tiles::tn_tile<D>(A, lda, B, ldb, blockIdx.x * 32, blockIdx.y * 32, m, n, r0, r1,
                    P + (int64_t)blockIdx.z * n * m, m);
}

// C (+)= A B, A tall (rows x k), B small (k x n); one 64 x 32 tile per block (128 threads).
template <class D>
__global__ void __launch_bounds__(128) k_gemm_nn(const D* __restrict__ A, int64_t lda, const D* __restrict__ B,
                                                 int64_t ldb, D* __restrict__ C, int64_t ldc, int64_t rows, int n,
                                                 int k, int accumulate) {
  tiles::nn_tile<D>(A, lda, B, ldb, C, ldc, rows, n, k, (int64_t)blockIdx.x * 64, blockIdx.y * 32, accumulate != 0);
}
}  // namespace bg
