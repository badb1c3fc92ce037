// BF16x3 complex products on the tcgen05 tensor cores (see gemm_tc.cuh).
//
// One CTA (256 threads, one per SM: 193 KB of shared memory) owns a 128 x 256 real
// output tile (128 rows, 128 complex columns) accumulated in FP32 in tensor memory
// (256 columns).  The K loop runs in stages of 32 complex (64 real) K values, double
// buffered: all threads load the FP64 operands (coalesced), split them into bf16 hi and
// lo parts and store them in the canonical K-major layout without swizzle (core matrices
// of 8 rows x 16 bytes; chunk c of every row at c * rows * 16 bytes, row groups of 8
// rows 128 bytes apart); one thread issues, per 16-wide K slice, the three products
// hi*hi, hi*lo, lo*hi (tcgen05.mma kind::f16, BF16 inputs, M = 128, N <= 256) and
// commits them to the stage's mbarrier, which the loaders wait on before they refill
// that stage.  The epilogue reads the accumulator with tcgen05.ld (warp w reads lanes
// 32 (w % 4) .. +31, column half w / 4) and writes FP32 partial tiles (kTN, split K)
// or the FP64 result (kNN).  Every mbarrier wait is bounded; on expiry the kernel sets
// the error word, waits (bounded) for its own MMAs, frees its tensor memory and returns.
#include "gemm_tc.cuh"

#include <cuda_bf16.h>

#include <algorithm>

namespace bg {
namespace tc {
namespace {

constexpr int kThreads = 256;
constexpr uint32_t kABytes = kTileM * kStepK * 2 * 2;   // 128 rows x 64 real K x 2 B = 16 KB
constexpr uint32_t kBBytes = kTileN * kStepK * 2 * 2;   // 256 rows x 64 real K x 2 B = 32 KB
constexpr uint32_t kAChunk = kTileM * 16;               // bytes of one 8-element K chunk of A
constexpr uint32_t kBChunk = kTileN * 16;
constexpr uint32_t kStageBytes = 2 * kABytes + 2 * kBBytes;
constexpr uint32_t kSmemBytes = 2 * kStageBytes + 1024;  // two stages, 1 KB for alignment
constexpr uint32_t kTmemCols = 256;
constexpr unsigned kWaitLimit = 1u << 24;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: K-major, no swizzle, start/LBO/SBO in 16-byte units,
// descriptor version 1 (bits 46-47).
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1), BF16 A and B
// (bits 7-9, 10-12 = 1), both K-major, N / 8 at bits 17-22, M / 16 at bits 24-28.
__device__ __forceinline__ uint32_t idesc(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kTileM >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
      "}\n" ::"r"(tmem),
      "l"(a), "l"(b), "r"(id), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  for (unsigned i = 0; i < kWaitLimit; ++i) {
    uint32_t ok;
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t"
        "}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

__device__ __forceinline__ uint32_t pack_bf16(double a, double b, uint32_t* lo) {
  const __nv_bfloat16 ha = __float2bfloat16_rn((float)a), hb = __float2bfloat16_rn((float)b);
  const __nv_bfloat16 la = __float2bfloat16_rn((float)(a - (double)__bfloat162float(ha)));
  const __nv_bfloat16 lb = __float2bfloat16_rn((float)(b - (double)__bfloat162float(hb)));
  *lo = (uint32_t)__bfloat16_as_ushort(la) | ((uint32_t)__bfloat16_as_ushort(lb) << 16);
  return (uint32_t)__bfloat16_as_ushort(ha) | ((uint32_t)__bfloat16_as_ushort(hb) << 16);
}

__device__ __forceinline__ void st16(uint32_t saddr, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(saddr), "r"(a), "r"(b), "r"(c), "r"(d) : "memory");
}

__device__ __forceinline__ double2 ldg2(const double2* p) { return __ldg(p); }

// The K range of split y of a kTN product (whole stages; the last split may be empty).
__device__ __host__ __forceinline__ void split_range(int K, int ksplit, int y, int* kb, int* ke) {
  int chunk = (K + ksplit - 1) / ksplit;
  chunk = (chunk + kStepK - 1) / kStepK * kStepK;
  *kb = min(K, y * chunk);
  *ke = min(K, *kb + chunk);
}

template <int MODE>
__global__ void __launch_bounds__(kThreads, 1)
    k_zgemm3(const ZDesc* __restrict__ descs, int ksplit, int max_m, int max_n, float* __restrict__ part, int* err) {
  const ZDesc d = descs[blockIdx.z];
  if (d.M <= 0 || d.N <= 0 || d.K <= 0) return;
  const int mt = (d.M + kTileM - 1) / kTileM, nt = (d.N + kTileN / 2 - 1) / (kTileN / 2);
  if ((int)blockIdx.x >= mt * nt) return;
  const int m0 = (blockIdx.x % mt) * kTileM, j0 = (blockIdx.x / mt) * (kTileN / 2);
  int kb = 0, ke = d.K;
  if (MODE == kTN) split_range(d.K, ksplit, blockIdx.y, &kb, &ke);
  if (ke <= kb) return;
  const int steps = (ke - kb + kStepK - 1) / kStepK;
  const int ncols = min(kTileN, 2 * (d.N - j0));          // real output columns of this tile
  const int nmma = (ncols + 15) / 16 * 16;

  extern __shared__ unsigned char dyn[];
  __shared__ __align__(8) uint64_t mbar[3];
  __shared__ uint32_t tmem_slot;
  __shared__ int s_fail;
  unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(dyn) + 1023) & ~(uintptr_t)1023);
  const uint32_t sbase = smem_addr(base);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (tid == 0) {
    mbar_init(smem_addr(&mbar[0]), 1);
    mbar_init(smem_addr(&mbar[1]), 1);
    mbar_init(smem_addr(&mbar[2]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_fail = 0;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  const uint32_t id = idesc(nmma);
  bool ok = true;

  for (int t = 0; t < steps; ++t) {
    const int stg = t & 1;
    const uint32_t sa_hi = sbase + stg * kStageBytes, sa_lo = sa_hi + kABytes;
    const uint32_t sb_hi = sa_hi + 2 * kABytes, sb_lo = sb_hi + kBBytes;
    if (t >= 2) {  // the MMAs of step t - 2 have released this stage (agreed by all threads)
      const bool expired = !mbar_wait(smem_addr(&mbar[stg]), ((t - 2) >> 1) & 1);
      if (__syncthreads_or(expired)) {
        ok = false;
        break;
      }
    }
    const int k0 = kb + t * kStepK;
    // loads first (32 independent 16-byte loads per thread), then split and store
    double2 va[4][4], vb[4][4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int p = tid + u * kThreads;
      const int r8 = p & 7, c = (p >> 3) & 7, g = p >> 6;
      const int i = m0 + 8 * g + r8;
      const int jl = 8 * g + r8, j = j0 + jl;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int k = k0 + 4 * c + q;
        const bool kin = k < ke;
        if (MODE == kTN)
          va[u][q] = (kin && i < d.M) ? ldg2(d.A + k + (int64_t)i * d.lda) : make_double2(0.0, 0.0);
        else
          va[u][q] = (kin && i < d.M) ? ldg2(d.A + i + (int64_t)k * d.lda) : make_double2(0.0, 0.0);
        vb[u][q] = (kin && j < d.N) ? ldg2(d.B + k + (int64_t)j * d.ldb) : make_double2(0.0, 0.0);
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int p = tid + u * kThreads;
      const int r8 = p & 7, c = (p >> 3) & 7, g = p >> 6;
      uint32_t h[4], l[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) h[q] = pack_bf16(va[u][q].x, va[u][q].y, &l[q]);
      const uint32_t offa = c * kAChunk + g * 128 + r8 * 16;
      st16(sa_hi + offa, h[0], h[1], h[2], h[3]);
      st16(sa_lo + offa, l[0], l[1], l[2], l[3]);
      // B rows 2 jl (real output part) and 2 jl + 1 (imaginary output part)
      uint32_t h0[4], l0[4], h1[4], l1[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const double re = vb[u][q].x, im = vb[u][q].y;
        if (MODE == kTN) {  // conj(a) b: (a_re, a_im) . (b_re, b_im) and (b_im, -b_re)
          h0[q] = pack_bf16(re, im, &l0[q]);
          h1[q] = pack_bf16(im, -re, &l1[q]);
        } else {            // a b: (b_re, -b_im) and (b_im, b_re)
          h0[q] = pack_bf16(re, -im, &l0[q]);
          h1[q] = pack_bf16(im, re, &l1[q]);
        }
      }
      const int r0 = 2 * (8 * g + r8), r1 = r0 + 1;
      const uint32_t offb0 = c * kBChunk + (r0 >> 3) * 128 + (r0 & 7) * 16;
      const uint32_t offb1 = c * kBChunk + (r1 >> 3) * 128 + (r1 & 7) * 16;
      st16(sb_hi + offb0, h0[0], h0[1], h0[2], h0[3]);
      st16(sb_lo + offb0, l0[0], l0[1], l0[2], l0[3]);
      st16(sb_hi + offb1, h1[0], h1[1], h1[2], h1[3]);
      st16(sb_lo + offb1, l1[0], l1[1], l1[2], l1[3]);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
      for (int s = 0; s < kStepK / 8; ++s) {  // 16 real K per slice: two chunks
        const uint64_t ah = sdesc(sa_hi + 2 * s * kAChunk, kAChunk, 128);
        const uint64_t al = sdesc(sa_lo + 2 * s * kAChunk, kAChunk, 128);
        const uint64_t bh = sdesc(sb_hi + 2 * s * kBChunk, kBChunk, 128);
        const uint64_t bl = sdesc(sb_lo + 2 * s * kBChunk, kBChunk, 128);
        mma_bf16(tmem, ah, bh, id, (t > 0 || s > 0) ? 1u : 0u);
        mma_bf16(tmem, ah, bl, id, 1u);
        mma_bf16(tmem, al, bh, id, 1u);
      }
      commit(smem_addr(&mbar[stg]));
    }
  }
  // every MMA issued so far done (bounded wait), then the accumulator is read
  if (tid == 0) {
    commit(smem_addr(&mbar[2]));
    if (!mbar_wait(smem_addr(&mbar[2]), 0)) s_fail = 1;
  }
  __syncthreads();
  if (!ok && tid == 0) s_fail = 1;
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (s_fail) {
    if (tid == 0) atomicExch(err, 1);
  } else {
    const int lg = warp & 3, half = warp >> 2;
    const int i = m0 + 32 * lg + lane;
    for (int cc = 0; cc < 8; ++cc) {
      const int n0 = half * 128 + cc * 16;
      if (n0 >= ncols) break;  // warp-uniform
      uint32_t r[16];
      const uint32_t taddr = tmem + ((uint32_t)(32 * lg) << 16) + (uint32_t)n0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
          "%15}, [%16];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (i < d.M) {
        if (MODE == kTN) {
          float* dst = part + (((size_t)blockIdx.z * ksplit + blockIdx.y) * max_m + i) * (2 * (size_t)max_n) +
                       2 * (size_t)j0 + n0;
#pragma unroll
          for (int q = 0; q < 16; ++q)
            if (n0 + q < ncols) dst[q] = __uint_as_float(r[q]);
        } else {
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const int j = j0 + (n0 >> 1) + q;
            if (2 * q < ncols - n0) {
              double2* cp = d.C + i + (int64_t)j * d.ldc;
              const double re = (double)__uint_as_float(r[2 * q]), im = (double)__uint_as_float(r[2 * q + 1]);
              if (d.op == kStore) {
                *cp = make_double2(re, im);
              } else {
                const double2 o = *cp;
                *cp = d.op == kAdd ? make_double2(o.x + re, o.y + im) : make_double2(o.x - re, o.y - im);
              }
            }
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

// C (op)= sum over the splits of the FP32 partial tiles, in split order, in FP64.
__global__ void k_zreduce(const ZDesc* __restrict__ descs, int ksplit, int max_m, int max_n,
                          const float* __restrict__ part) {
  const ZDesc d = descs[blockIdx.y];
  if (d.M <= 0 || d.N <= 0 || d.K <= 0) return;
  int used = 0;
  for (int y = 0; y < ksplit; ++y) {
    int kb, ke;
    split_range(d.K, ksplit, y, &kb, &ke);
    if (ke > kb) used = y + 1;
  }
  const int64_t total = (int64_t)d.M * d.N;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(t % d.M), j = (int)(t / d.M);
    double re = 0.0, im = 0.0;
    for (int y = 0; y < used; ++y) {
      const float* p = part + (((size_t)blockIdx.y * ksplit + y) * max_m + i) * (2 * (size_t)max_n) + 2 * (size_t)j;
      re += (double)p[0];
      im += (double)p[1];
    }
    double2* cp = d.C + i + (int64_t)j * d.ldc;
    if (d.op == kStore) {
      *cp = make_double2(re, im);
    } else {
      const double2 o = *cp;
      *cp = d.op == kAdd ? make_double2(o.x + re, o.y + im) : make_double2(o.x - re, o.y - im);
    }
  }
}

}  // namespace

cudaError_t prepare_zgemm() {
  cudaError_t e = cudaFuncSetAttribute((const void*)k_zgemm3<kTN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kSmemBytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void*)k_zgemm3<kNN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes);
  return e;
}

int tn_ksplit(int ndesc, int max_m, int max_n, int max_k) {
  const int tiles = ((max_m + kTileM - 1) / kTileM) * ((max_n + kTileN / 2 - 1) / (kTileN / 2)) * std::max(ndesc, 1);
  int ks = (2 * 148 + tiles - 1) / tiles;
  const int max_split = std::max(1, (max_k + 8 * kStepK - 1) / (8 * kStepK));  // at least 8 stages each
  return std::max(1, std::min(ks, max_split));
}

int launch_zgemm(int mode, const ZDesc* d_desc, int ndesc, int max_m, int max_n, int max_k, int ksplit, float* work,
                 int* err, cudaStream_t s) {
  const unsigned tiles =
      (unsigned)(((max_m + kTileM - 1) / kTileM) * ((max_n + kTileN / 2 - 1) / (kTileN / 2)));
  if (tiles == 0 || ndesc == 0) return 0;
  (void)max_k;
  if (mode == kTN) {
    k_zgemm3<kTN><<<dim3(tiles, (unsigned)ksplit, (unsigned)ndesc), kThreads, kSmemBytes, s>>>(d_desc, ksplit, max_m,
                                                                                               max_n, work, err);
    const int64_t total = (int64_t)max_m * max_n;
    const unsigned blocks = (unsigned)std::min<int64_t>((total + 255) / 256, 1024);
    k_zreduce<<<dim3(blocks, (unsigned)ndesc), 256, 0, s>>>(d_desc, ksplit, max_m, max_n, work);
    return 2;
  }
  k_zgemm3<kNN><<<dim3(tiles, 1, (unsigned)ndesc), kThreads, kSmemBytes, s>>>(d_desc, 1, max_m, max_n, nullptr, err);
  return 1;
}

}  // namespace tc
}  // namespace bg

// ------------------------------------------------------------------ C ABI
#include <string>

#include "op_internal.h"

using namespace bg;

extern "C" int bg_zgemm_bf16x3(bg_ctx* ctx, int32_t mode, int64_t m, int64_t n, int64_t k, const double* a,
                               int64_t lda, const double* b, int64_t ldb, double* c, int64_t ldc, int32_t op,
                               void* stream) {
  if (!ctx) return fail(nullptr, BG_EINVAL, "null context");
  if (mode != tc::kTN && mode != tc::kNN) return fail(ctx, BG_EINVAL, "mode must be 0 (A^H B) or 1 (A B)");
  if (op < tc::kStore || op > tc::kSub) return fail(ctx, BG_EINVAL, "op must be 0 (=), 1 (+=) or 2 (-=)");
  if (m < 0 || n < 0 || k < 0 || m > (1 << 30) || n > (1 << 20) || k > (1 << 30))
    return fail(ctx, BG_ESHAPE, "dimensions out of range");
  if (m == 0 || n == 0) return BG_OK;
  if (!a || !b || !c) return fail(ctx, BG_EINVAL, "null matrix");
  const int64_t arows = mode == tc::kTN ? k : m;
  if (lda < std::max<int64_t>(arows, 1) || ldb < std::max<int64_t>(k, 1) || ldc < m)
    return fail(ctx, BG_ESHAPE, "leading dimensions too small");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
  if ((e = tc::prepare_zgemm()) != cudaSuccess) return cuda_fail(ctx, e, "tensor-core product attributes");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  tc::ZDesc d{reinterpret_cast<const double2*>(a), reinterpret_cast<const double2*>(b), reinterpret_cast<double2*>(c),
              lda, ldb, ldc, (int)m, (int)n, (int)k, op};
  if (k == 0) {
    if (op != tc::kStore) return BG_OK;
    e = cudaMemset2DAsync(c, ldc * 2 * sizeof(double), 0, m * 2 * sizeof(double), n, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? BG_OK : cuda_fail(ctx, e, "zero product");
  }
  const int ks = mode == tc::kTN ? tc::tn_ksplit(1, (int)m, (int)n, (int)k) : 1;
  tc::ZDesc* dd = nullptr;
  int* derr = nullptr;
  float* work = nullptr;
  const size_t wf = mode == tc::kTN ? tc::tn_workspace_floats(1, ks, (int)m, (int)n) : 0;
  e = cudaMalloc(&dd, sizeof(tc::ZDesc));
  if (e == cudaSuccess) e = cudaMalloc(&derr, sizeof(int));
  if (e == cudaSuccess && wf) e = cudaMalloc(&work, wf * sizeof(float));
  int herr = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(dd, &d, sizeof d, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(derr, 0, sizeof(int), s);
  if (e == cudaSuccess) {
    tc::launch_zgemm(mode, dd, 1, (int)m, (int)n, (int)k, ks, work, derr, s);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(dd);
  cudaFree(derr);
  if (work) cudaFree(work);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "tensor-core product");
  if (herr) return fail(ctx, BG_ETIMEOUT, "tensor-core product: a pipeline wait gave up");
  return BG_OK;
}
