// FP64 tall-skinny products (real double or complex double2) with shared-memory tiles
// filled by cp.async ahead of the arithmetic.  tcgen05 has no FP64 kind; the FP64 tensor
// path of sm_100a is mma.sync m8n8k4 f64 (DMMA), whose peak matches the CUDA cores' DFMA
// (37 TFLOP/s measured against 34 for a DFMA loop on one B200) but which issues 256
// multiply-adds per warp instruction instead of 32, so the hot tiles use it.
//   tn_tile / nn_tile (DFMA, 4 x 4 register tiles): the small generic products
//     (32 x 32 Gram tiles, 64 x 32 rotation tiles)
//   tn_tile48_mma: P = A^H B, 48 x 48 tiles (projections P^H X, Davidson Grams)
//   nn_tile64_mma: C (+)= A B, 64 x 64 tiles (back-projection P W, Davidson rotations)
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

// 48 x 48 tiles of P = A^H B for the Davidson's Grams and the projections (m, n up to the
// basis capacity or the projector count): the rows stream through shared-memory stages of
// kBK48 rows each, filled by cp.async ahead of the arithmetic.
constexpr int kBK48 = 32;

// tn_tile48_mma: P[j * ldp + i] = sum over rows r0 .. r1 - 1 of conj(A[r][i0 + i]) B[r][j0 + j]
// for the valid i < m - i0, j < n - j0, with mma.sync m8n8k4 f64 (DMMA) on fragments read
// from shared memory.  One DMMA does 256 multiply-adds per warp instruction against 32
// for DFMA, so the FP64 pipe is no longer held back by issue slots and operand reads.
// 256 threads = 8 warps: warp w takes the K half g = w / 4 of every 32-row stage (four
// k-steps of 4 rows each) and the 24 x 24 output block (wi, wj) = ((w / 2) % 2, w % 2),
// 3 x 3 MMA tiles of 8 x 8; the two halves' sums meet in shared memory at the end (half 1
// stores, half 0 adds and writes P).  Two stages, double buffered: 32-row stages give each
// warp four k-steps per barrier (16-row stages with three buffers measured 11.16 against
// 9.63 ms for the Si216 projection) and still fit two CTAs per SM.  A stage holds each
// column's 32 rows with a pitch of 36 elements, so the fragment reads (8 columns x 4 rows
// per warp) meet no bank conflicts for double and double2.  Fragments of m8n8k4 (row.col,
// f64): A (8 x 4) lane holds (m, k) = (lane / 4, lane % 4); B (4 x 8) (k, n) = (lane % 4,
// lane / 4); C (8 x 8) (m, n) = (lane / 4, 2 (lane % 4) + e), e = 0, 1.  Complex:
// Re += ar br + ai bi, Im += ar bi - ai br (four real DMMAs; A^H conjugates A).
constexpr int kStagesM = 2;
constexpr int kPitchM = kBK48 + 4;
constexpr int kPitchNB = kBK + 4;  // nn_tile64_mma's B columns
template <class D>
constexpr size_t tn48m_smem_bytes() {
  return (size_t)2 * kStagesM * 48 * kPitchM * sizeof(D);
}
__device__ __forceinline__ void dmma8x8x4(double& c0, double& c1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
      : "+d"(c0), "+d"(c1)
      : "d"(a), "d"(b));
}
template <class D>
__device__ __forceinline__ void tn_tile48_mma(const D* __restrict__ A, int64_t lda, const D* __restrict__ B,
                                              int64_t ldb, int i0, int j0, int m, int n, int64_t r0, int64_t r1,
                                              D* __restrict__ P, int64_t ldp) {
  constexpr bool kComplex = sizeof(D) == 16;
  extern __shared__ __align__(16) unsigned char tn48_smem[];
  D* As = reinterpret_cast<D*>(tn48_smem);  // [stage][48 columns][kPitchM rows]
  D* Bs = As + kStagesM * 48 * kPitchM;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = warp >> 2, wi = (warp >> 1) & 1, wj = warp & 1;
  const int fm = lane >> 2, fk = lane & 3;
  const bool warp_live = i0 + 24 * wi < m && j0 + 24 * wj < n;
  double cre[3][3][2], cim[3][3][2];
#pragma unroll
  for (int x = 0; x < 3; ++x)
#pragma unroll
    for (int y = 0; y < 3; ++y)
#pragma unroll
      for (int e = 0; e < 2; ++e) cre[x][y][e] = cim[x][y][e] = 0.0;
  auto load = [&](int buf, int64_t rb) {
    for (int e = tid; e < 2 * 48 * kBK48; e += 256) {
      const int mat = e / (48 * kBK48), idx = e - mat * (48 * kBK48);
      const int rr = idx % kBK48, c = idx / kBK48;
      const int64_t r = rb + rr;
      D* dst = (mat == 0 ? As : Bs) + (buf * 48 + c) * kPitchM + rr;
      const bool ok = r < r1 && (mat == 0 ? i0 + c < m : j0 + c < n);
      if (ok)
        async_copy(dst, mat == 0 ? A + (int64_t)(i0 + c) * lda + r : B + (int64_t)(j0 + c) * ldb + r);
      else
        *dst = Arith<D>::zero();
    }
    async_commit();
  };
  const int64_t steps = (r1 - r0 + kBK48 - 1) / kBK48;
  // one cp.async group per stage, empty ones past the end (as in tn_tile48)
#pragma unroll
  for (int s = 0; s < kStagesM - 1; ++s) {
    if (s < steps)
      load(s, r0 + s * kBK48);
    else
      async_commit();
  }
  for (int64_t s = 0; s < steps; ++s) {
    async_wait<kStagesM - 2>();
    __syncthreads();  // stage s visible to all; every warp is done with stage s - 1
    const int64_t nxt = s + kStagesM - 1;
    if (nxt < steps)
      load((int)(nxt % kStagesM), r0 + nxt * kBK48);  // refills the buffer of stage s - 1
    else
      async_commit();
    if (warp_live) {
      const D* as = As + (int)(s % kStagesM) * 48 * kPitchM + (24 * wi + fm) * kPitchM + (kBK48 / 2) * g + fk;
      const D* bs = Bs + (int)(s % kStagesM) * 48 * kPitchM + (24 * wj + fm) * kPitchM + (kBK48 / 2) * g + fk;
#pragma unroll
      for (int kk = 0; kk < kBK48 / 8; ++kk) {
        D a[3], b[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          a[q] = as[8 * q * kPitchM + 4 * kk];
          b[q] = bs[8 * q * kPitchM + 4 * kk];
        }
#pragma unroll
        for (int x = 0; x < 3; ++x)
#pragma unroll
          for (int y = 0; y < 3; ++y) {
            if constexpr (kComplex) {
              dmma8x8x4(cre[x][y][0], cre[x][y][1], a[x].x, b[y].x);
              dmma8x8x4(cre[x][y][0], cre[x][y][1], a[x].y, b[y].y);
              dmma8x8x4(cim[x][y][0], cim[x][y][1], a[x].x, b[y].y);
              dmma8x8x4(cim[x][y][0], cim[x][y][1], -a[x].y, b[y].x);
            } else {
              dmma8x8x4(cre[x][y][0], cre[x][y][1], a[x], b[y]);
            }
          }
      }
    }
  }
  async_wait<0>();
  __syncthreads();  // every stage consumed: the A stages hold the K halves' meeting place
  D* red = As;      // [48 columns][48 rows] of the tile, local indices
  if (g == 1 && warp_live) {
#pragma unroll
    for (int x = 0; x < 3; ++x)
#pragma unroll
      for (int y = 0; y < 3; ++y)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int i = 24 * wi + 8 * x + fm, j = 24 * wj + 8 * y + 2 * fk + e;
          if constexpr (kComplex)
            red[j * 48 + i] = make_double2(cre[x][y][e], cim[x][y][e]);
          else
            red[j * 48 + i] = cre[x][y][e];
        }
  }
  __syncthreads();
  if (g == 0 && warp_live) {
#pragma unroll
    for (int x = 0; x < 3; ++x)
#pragma unroll
      for (int y = 0; y < 3; ++y)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int i = 24 * wi + 8 * x + fm, j = 24 * wj + 8 * y + 2 * fk + e;
          if (i0 + i < m && j0 + j < n) {
            const D h = red[j * 48 + i];
            if constexpr (kComplex)
              P[(int64_t)(j0 + j) * ldp + i0 + i] = make_double2(cre[x][y][e] + h.x, cim[x][y][e] + h.y);
            else
              P[(int64_t)(j0 + j) * ldp + i0 + i] = cre[x][y][e] + h;
          }
        }
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

// 64 x 64 tiles of C (+)= A B, A tall (rows x k, column-major), B small (k x n): the inner
// index streams through kStages64 shared-memory stages of kBK entries, filled by cp.async
// kStages64 - 1 stages ahead.
constexpr int kStages64 = 3;

// nn_tile64_mma: C (+)= A B for one 64 x 64 tile (rows r0 .., columns j0 ..) with
// mma.sync m8n8k4 f64.  8 warps: warp w owns rows r0 + 32 (w % 2) ..
// + 31 and columns j0 + 16 (w / 2) .. + 15, 4 x 2 MMA tiles of 8 x 8; each 16-entry
// stage is 4 k-steps of 4.  Shared memory holds A's stage rows with a pitch of 66
// (complex) or 68 (real) elements and B's columns with a pitch of 20, so the fragment
// reads (A: 8 rows x 4 inner indices; B: 4 inner indices x 8 columns) meet no bank
// conflicts.  Complex: Re += ar br - ai bi, Im += ar bi + ai br.  SKIP_EMPTY skips the
// warps whose 16 columns lie at or beyond n.  Dynamic shared memory: nn64m_smem_bytes<D>().
template <class D>
__host__ __device__ constexpr int nn_pitch_a() {
  return sizeof(D) == 16 ? 66 : 68;
}
template <class D>
constexpr size_t nn64m_smem_bytes() {
  return (size_t)kStages64 * (kBK * nn_pitch_a<D>() + 64 * kPitchNB) * sizeof(D);
}
template <class D, bool SKIP_EMPTY = false>
__device__ __forceinline__ void nn_tile64_mma(const D* __restrict__ A, int64_t lda, const D* __restrict__ B,
                                              int64_t ldb, D* __restrict__ C, int64_t ldc, int64_t rows, int n,
                                              int k, int64_t r0, int j0, bool accumulate) {
  constexpr bool kComplex = sizeof(D) == 16;
  constexpr int PA = nn_pitch_a<D>();
  extern __shared__ __align__(16) unsigned char nn64_smem[];
  D* As = reinterpret_cast<D*>(nn64_smem);  // [stage][kBK][PA]: 64 rows of A per inner index
  D* Bs = As + kStages64 * kBK * PA;        // [stage][64 columns][kPitchNB]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wr = warp & 1, wc = warp >> 1;
  const int fm = lane >> 2, fk = lane & 3;
  const bool live = !SKIP_EMPTY || j0 + 16 * wc < n;
  double cre[4][2][2], cim[4][2][2];
#pragma unroll
  for (int x = 0; x < 4; ++x)
#pragma unroll
    for (int y = 0; y < 2; ++y)
#pragma unroll
      for (int e = 0; e < 2; ++e) cre[x][y][e] = cim[x][y][e] = 0.0;
  auto load = [&](int buf, int pb) {
    D* as = As + buf * kBK * PA;
    D* bs = Bs + buf * 64 * kPitchNB;
#pragma unroll
    for (int q = 0; q < 4; ++q) {  // A: kBK x 64, consecutive threads on consecutive rows
      const int e = tid + 256 * q;
      const int rr = e & 63, p = e >> 6;
      const int64_t r = r0 + rr;
      D* d = as + p * PA + rr;
      if (r < rows && pb + p < k)
        async_copy(d, A + (int64_t)(pb + p) * lda + r);
      else
        *d = Arith<D>::zero();
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {  // B: 64 columns x kBK, consecutive threads on consecutive entries
      const int e = tid + 256 * q;
      const int p = e & (kBK - 1), c = e >> 4;
      D* d = bs + c * kPitchNB + p;
      if (pb + p < k && j0 + c < n)
        async_copy(d, B + (int64_t)(j0 + c) * ldb + pb + p);
      else
        *d = Arith<D>::zero();
    }
    async_commit();
  };
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
    __syncthreads();  // stage s visible to all; every warp is done with stage s - 1
    const int nxt = s + kStages64 - 1;
    if (nxt < steps)
      load(nxt % kStages64, nxt * kBK);  // refills the buffer of stage s - 1
    else
      async_commit();
    if (live) {
      const D* as = As + (s % kStages64) * kBK * PA + fk * PA + 32 * wr + fm;
      const D* bs = Bs + (s % kStages64) * 64 * kPitchNB + (16 * wc + fm) * kPitchNB + fk;
#pragma unroll
      for (int kk = 0; kk < kBK / 4; ++kk) {
        D a[4], b[2];
#pragma unroll
        for (int q = 0; q < 4; ++q) a[q] = as[4 * kk * PA + 8 * q];
#pragma unroll
        for (int q = 0; q < 2; ++q) b[q] = bs[8 * q * kPitchNB + 4 * kk];
#pragma unroll
        for (int x = 0; x < 4; ++x)
#pragma unroll
          for (int y = 0; y < 2; ++y) {
            if constexpr (kComplex) {
              dmma8x8x4(cre[x][y][0], cre[x][y][1], a[x].x, b[y].x);
              dmma8x8x4(cre[x][y][0], cre[x][y][1], -a[x].y, b[y].y);
              dmma8x8x4(cim[x][y][0], cim[x][y][1], a[x].x, b[y].y);
              dmma8x8x4(cim[x][y][0], cim[x][y][1], a[x].y, b[y].x);
            } else {
              dmma8x8x4(cre[x][y][0], cre[x][y][1], a[x], b[y]);
            }
          }
      }
    }
  }
  async_wait<0>();
  if (!live) return;
#pragma unroll
  for (int x = 0; x < 4; ++x)
#pragma unroll
    for (int y = 0; y < 2; ++y)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int64_t r = r0 + 32 * wr + 8 * x + fm;
        const int j = j0 + 16 * wc + 8 * y + 2 * fk + e;
        if (r < rows && j < n) {
          D v;
          if constexpr (kComplex)
            v = make_double2(cre[x][y][e], cim[x][y][e]);
          else
            v = cre[x][y][e];
          D& out = C[(int64_t)j * ldc + r];
          out = accumulate ? Arith<D>::add(out, v) : v;
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
