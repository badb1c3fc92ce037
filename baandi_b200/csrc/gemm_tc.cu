// BF16x3 complex products on the tcgen05 tensor cores (see gemm_tc.cuh).
//
// Split pass (k_split_*): one thread per (source column, K tile) reads 16 complex FP64
// values (a K run of a column for kTN operands and B, a row across 16 columns for the kNN
// A operand, whose rows are contiguous across neighbouring threads), rounds them to
// FP32, forms the variants the real product needs and writes their bf16 hi and lo
// chunks; neighbouring threads write neighbouring 16-byte chunks.
//
// Product pass (k_tc3): one CTA of 128 threads owns a 128 x trb real output tile (trb <=
// 256 real columns, 128 complex) accumulated in FP32 in tensor memory.  Its K range
// streams through a ring of kStages shared-memory stages (an A tile of 16 KB and a B tile
// of trb x 128 bytes each): thread 0 waits for a stage to be free (its `empty` mbarrier,
// signalled by tcgen05.commit), arms the stage's `full` mbarrier with the byte count and
// issues two cp.async.bulk copies of the contiguous panel tiles; thread 32 waits on
// `full`, issues per 16-wide K slice the three products hi*hi, hi*lo, lo*hi
// (tcgen05.mma kind::f16, BF16 inputs, M = 128, N = trb) and commits them to `empty`.
// After the last stage a commit to `done` releases the epilogue: warp w reads TMEM lanes
// 32 w .. 32 w + 31 with tcgen05.ld and writes FP32 partial tiles (kTN, split K) or the
// FP64 result (kNN).  Every mbarrier wait is bounded; on expiry the kernel sets the
// error word, waits (bounded) for its own copies and MMAs in flight, frees its tensor
// memory and returns.  No copy is multicast; the sources are this GPU's own memory.
#include "gemm_tc.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <cstdio>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

namespace bg {
namespace tc {
namespace {

constexpr int kThreads = 128;
constexpr int kStages = 4;
constexpr unsigned kWaitLimit = 1u << 24;
constexpr int kSms = 148;
constexpr int kMaxChain = 256;  // K tiles accumulated by one CTA of a split-K product

enum : int { kVarA = 0, kVarTnB = 1, kVarNnB = 2 };

__host__ __device__ __forceinline__ size_t tile_bytes_d(int rows) { return (size_t)rows * kStepK * 4; }
__host__ __device__ __forceinline__ int k_tiles_d(int64_t k) { return (int)((2 * k + kStepK - 1) / kStepK); }

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

__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
  asm volatile(
      "{\n\t"
      ".reg .b64 st;\n\t"
      "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t"
      "}\n" ::"r"(mbar),
      "r"(bytes)
      : "memory");
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

// Global -> shared bulk copy (16-byte aligned addresses, size a multiple of 16) that
// completes its bytes on the stage's mbarrier.
__device__ __forceinline__ void bulk_copy(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(mbar)
               : "memory");
}

// The K-tile range of split y (the last splits may be empty).
__device__ __host__ __forceinline__ void split_range(int ktd, int ksplit, int y, int* kb, int* ke) {
  const int chunk = (ktd + ksplit - 1) / ksplit;
  *kb = min(ktd, y * chunk);
  *ke = min(ktd, *kb + chunk);
}

// ------------------------------------------------------------------ split pass
// Source of a split: element (panel column j, complex K index k) at X[k sk + j sj];
// panel row nvar j + v holds variant v of column j.
struct SplitArgs {
  const double2* X;
  int64_t sk, sj;
  int cols, K;
  int nvar, var;
  int R;    // rows per tile
  int ktc;  // K tiles of the panel layout (row tile stride)
  unsigned char* panel;
};

// bf16 pair (a, b) rounded to nearest, and the remainders a - hi, b - hi.
__device__ __forceinline__ uint32_t bf2(float a, float b, float* ra, float* rb) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  const float2 f = __bfloat1622float2(h);
  *ra = a - f.x;
  *rb = b - f.y;
  return *reinterpret_cast<const uint32_t*>(&h);
}

// One thread per (source column j of the row tile, K tile): its 16 complex values (a
// 256-byte run of the column, or one row across 16 columns for the kNN A operand) are
// loaded together, then every variant row nvar j + v gets its four hi and four lo
// chunks; neighbouring threads take neighbouring columns, so each chunk store of a warp
// is contiguous.
__device__ __forceinline__ void split_tile_rows(const SplitArgs& a, int rt, int64_t first, int64_t step) {
  const int ktd = k_tiles_d(a.K);
  const int R = a.R, per = R / a.nvar;  // source columns per row tile
  const int64_t items = (int64_t)ktd * per;
  for (int64_t idx = first; idx < items; idx += step) {
    const int kt = (int)(idx / per);
    const int jl = (int)(idx - (int64_t)kt * per);
    const int j = rt * per + jl;
    const int k0 = kt * (kStepK / 2);
    double2 x[16];
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      x[u] = make_double2(0.0, 0.0);
      if (j < a.cols && k0 + u < a.K) x[u] = __ldg(a.X + (int64_t)(k0 + u) * a.sk + (int64_t)j * a.sj);
    }
    unsigned char* tile = a.panel + ((size_t)rt * a.ktc + kt) * tile_bytes_d(R);
    for (int v = 0; v < a.nvar; ++v) {
      const int r = jl * a.nvar + v;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        float f[8];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const float re = (float)x[4 * c + u].x, im = (float)x[4 * c + u].y;
          float p0 = re, p1 = im;
          if (a.var == kVarTnB && v == 1) {  // conj(a) b, imaginary output part: (b_im, -b_re)
            p0 = im;
            p1 = -re;
          } else if (a.var == kVarNnB) {     // a b: (b_re, -b_im) and (b_im, b_re)
            if (v == 0) {
              p1 = -im;
            } else {
              p0 = im;
              p1 = re;
            }
          }
          f[2 * u] = p0;
          f[2 * u + 1] = p1;
        }
        uint4 hi, lo;
        float l[8], rest[8];
        hi.x = bf2(f[0], f[1], &l[0], &l[1]);
        hi.y = bf2(f[2], f[3], &l[2], &l[3]);
        hi.z = bf2(f[4], f[5], &l[4], &l[5]);
        hi.w = bf2(f[6], f[7], &l[6], &l[7]);
        lo.x = bf2(l[0], l[1], &rest[0], &rest[1]);
        lo.y = bf2(l[2], l[3], &rest[2], &rest[3]);
        lo.z = bf2(l[4], l[5], &rest[4], &rest[5]);
        lo.w = bf2(l[6], l[7], &rest[6], &rest[7]);
        const size_t q = (size_t)c * R + r;  // chunk c of row r
        *reinterpret_cast<uint4*>(tile + 16 * q) = hi;
        *reinterpret_cast<uint4*>(tile + (size_t)R * 64 + 16 * q) = lo;
      }
    }
  }
}

__device__ __forceinline__ SplitArgs split_of(const ZDesc& d, int mode, int which, int R, int ktc,
                                              unsigned char* panel) {
  SplitArgs a;
  a.K = d.K;
  a.R = R;
  a.ktc = ktc;
  a.panel = panel;
  if (which == 0) {
    a.X = d.A;
    a.cols = d.M;
    a.nvar = 1;
    a.var = kVarA;
    if (mode == kTN) {
      a.sk = 1;
      a.sj = d.lda;
    } else {
      a.sk = d.lda;
      a.sj = 1;
    }
  } else {
    a.X = d.B;
    a.cols = d.N;
    a.nvar = 2;
    a.var = mode == kTN ? kVarTnB : kVarNnB;
    a.sk = 1;
    a.sj = d.ldb;
  }
  return a;
}

// Split of operand `which` (0: A, 1: B) of every descriptor; blockIdx.y = row tile,
// blockIdx.z = descriptor.
__global__ void k_split_desc(const ZDesc* __restrict__ descs, int mode, int which, int R, int ktc, size_t stride,
                             unsigned char* base) {
  const ZDesc d = descs[blockIdx.z];
  if (d.M <= 0 || d.N <= 0 || d.K <= 0) return;
  if (which == 0 && d.a_split) return;
  const SplitArgs a = split_of(d, mode, which, R, ktc, base + blockIdx.z * stride);
  const int row_tiles = (a.nvar * a.cols + R - 1) / R;
  if ((int)blockIdx.y >= row_tiles) return;
  split_tile_rows(a, blockIdx.y, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, (int64_t)gridDim.x * blockDim.x);
}

__global__ void k_split_args(SplitArgs a) {
  split_tile_rows(a, blockIdx.y, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, (int64_t)gridDim.x * blockDim.x);
}

unsigned split_blocks(int64_t items) {
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(1024, (items + 256 * 2 - 1) / (256 * 2)));
}

// ------------------------------------------------------------------ product pass
struct Geo {
  int ktc;  // K tiles of the launch's own panels
  int trb;  // B tile rows
  int ksplit;
  int max_m, max_n;
  size_t a_stride, b_stride;
};

__host__ __device__ __forceinline__ uint32_t stage_bytes(int trb) {
  return (uint32_t)(tile_bytes_d(kTileM) + tile_bytes_d(trb));
}
inline size_t smem_bytes(int trb) { return (size_t)kStages * stage_bytes(trb) + 1024; }

template <int MODE>
__global__ void __launch_bounds__(kThreads, 1)
    k_tc3(const ZDesc* __restrict__ descs, Geo g, const unsigned char* __restrict__ apan,
          const unsigned char* __restrict__ bpan, float* __restrict__ part, int* err) {
  const ZDesc d = descs[blockIdx.z];
  if (d.M <= 0 || d.N <= 0 || d.K <= 0) return;
  const int nr = 2 * d.N;
  const int mt_n = (d.M + kTileM - 1) / kTileM, nt_n = (nr + g.trb - 1) / g.trb;
  if ((int)blockIdx.x >= mt_n * nt_n) return;
  // CTAs that share an A tile (the large operand of kNN) are neighbours in launch order
  const int mt = blockIdx.x / nt_n, nt = blockIdx.x % nt_n;
  const int ktd = k_tiles_d(d.K);
  int kb = 0, ke = ktd;
  if (MODE == kTN) split_range(ktd, g.ksplit, blockIdx.y, &kb, &ke);
  if (ke <= kb) return;
  if (!d.a_split && g.a_stride == 0) {  // a launch for presplit A given a descriptor without its panel
    if (threadIdx.x == 0) atomicExch(err, 2);
    return;
  }
  const int steps = ke - kb;
  const int ncols = min(g.trb, nr - nt * g.trb);  // real output columns of this tile
  const int nmma = (ncols + 15) / 16 * 16;
  const uint32_t abytes = (uint32_t)tile_bytes_d(kTileM), bbytes = (uint32_t)tile_bytes_d(g.trb);
  const unsigned char* a_src = d.a_split ? d.a_split + ((size_t)mt * d.a_kt + kb) * abytes
                                         : apan + blockIdx.z * g.a_stride + ((size_t)mt * g.ktc + kb) * abytes;
  const unsigned char* b_src = bpan + blockIdx.z * g.b_stride + ((size_t)nt * g.ktc + kb) * bbytes;

  extern __shared__ unsigned char dyn[];
  __shared__ __align__(8) uint64_t full[kStages], empty[kStages], done;
  __shared__ uint32_t tmem_slot;
  __shared__ int s_fail, s_issued, s_consumed;
  unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(dyn) + 1023) & ~(uintptr_t)1023);
  const uint32_t sbase = smem_addr(base);
  const uint32_t sstage = stage_bytes(g.trb);
  // tensor-memory columns: the accumulator's trb, rounded up to a power of two >= 32
  uint32_t tcols = 32;
  while (tcols < (uint32_t)g.trb) tcols <<= 1;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(smem_addr(&full[s]), 1);
      mbar_init(smem_addr(&empty[s]), 1);
    }
    mbar_init(smem_addr(&done), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_fail = 0;
    s_issued = 0;
    s_consumed = 0;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                 "r"(tcols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;

  if (tid == 0) {  // producer
    int t = 0;
    for (; t < steps; ++t) {
      const int s = t % kStages;
      if (t >= kStages && !mbar_wait(smem_addr(&empty[s]), (uint32_t)((t / kStages - 1) & 1))) {
        s_fail = 1;
        break;
      }
      const uint32_t sa = sbase + s * sstage, sb = sa + abytes;
      mbar_expect_tx(smem_addr(&full[s]), abytes + bbytes);
      bulk_copy(sa, a_src + (size_t)t * abytes, abytes, smem_addr(&full[s]));
      bulk_copy(sb, b_src + (size_t)t * bbytes, bbytes, smem_addr(&full[s]));
    }
    s_issued = t;
  } else if (tid == 32) {  // MMA issuer
    const uint32_t id = idesc(nmma);
    int t = 0;
    for (; t < steps; ++t) {
      const int s = t % kStages;
      if (!mbar_wait(smem_addr(&full[s]), (uint32_t)((t / kStages) & 1))) {
        s_fail = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t sa = sbase + s * sstage, sb = sa + abytes;
      const uint32_t alo = sa + kTileM * 64, blo = sb + (uint32_t)g.trb * 64;
      const uint32_t achunk = kTileM * 16, bchunk = (uint32_t)g.trb * 16;
#pragma unroll
      for (int sl = 0; sl < kStepK / 16; ++sl) {  // 16 real K per MMA: two 8-value chunks
        const uint64_t ah = sdesc(sa + 2 * sl * achunk, achunk, 128);
        const uint64_t al = sdesc(alo + 2 * sl * achunk, achunk, 128);
        const uint64_t bh = sdesc(sb + 2 * sl * bchunk, bchunk, 128);
        const uint64_t bl = sdesc(blo + 2 * sl * bchunk, bchunk, 128);
        mma_bf16(tmem, ah, bh, id, (t > 0 || sl > 0) ? 1u : 0u);
        mma_bf16(tmem, ah, bl, id, 1u);
        mma_bf16(tmem, al, bh, id, 1u);
      }
      commit(smem_addr(&empty[s]));
    }
    s_consumed = t;
    commit(smem_addr(&done));  // every MMA issued above
  }
  __syncthreads();
  if (tid == 32) {
    if (!mbar_wait(smem_addr(&done), 0)) s_fail = 1;
  }
  if (tid == 0) {  // copies issued but never consumed (a failed wait): let them land
    for (int t = s_consumed; t < s_issued; ++t)
      if (!mbar_wait(smem_addr(&full[t % kStages]), (uint32_t)((t / kStages) & 1))) s_fail = 1;
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (s_fail) {
    if (tid == 0) atomicExch(err, 1);
  } else {
    const int i = mt * kTileM + 32 * warp + lane;
    const bool row = i < d.M;
    // batches of 64 real columns: for += and -= the batch's 32 complex C values are loaded
    // together (all in flight) before its accumulator columns are read
    for (int nb = 0; nb < ncols; nb += 64) {
      double2 o[32];
      if (MODE == kNN && d.op != kStore && row) {
#pragma unroll
        for (int q = 0; q < 32; ++q)
          if (nb + 2 * q < ncols) o[q] = d.C[i + (int64_t)((nt * g.trb + nb) / 2 + q) * d.ldc];
      }
#pragma unroll
      for (int sub = 0; sub < 4; ++sub) {
        const int n0 = nb + 16 * sub;
        if (n0 >= ncols) break;  // warp-uniform
        uint32_t r[16];
        const uint32_t taddr = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)n0;
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
            "%14, %15}, [%16];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (!row) continue;
        const int c0 = nt * g.trb + n0;  // real output column of r[0]
        if (MODE == kTN) {
          float* dst = part + (((size_t)blockIdx.z * g.ksplit + blockIdx.y) * g.max_m + i) * (2 * (size_t)g.max_n) + c0;
#pragma unroll
          for (int q = 0; q < 16; ++q)
            if (n0 + q < ncols) dst[q] = __uint_as_float(r[q]);
        } else {
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            if (n0 + 2 * q >= ncols) break;
            const int j = (c0 >> 1) + q;
            const double re = (double)__uint_as_float(r[2 * q]), im = (double)__uint_as_float(r[2 * q + 1]);
            double2 v = make_double2(re, im);
            if (d.op != kStore) {
              const double2 old = o[8 * sub + q];
              v = d.op == kAdd ? make_double2(old.x + re, old.y + im) : make_double2(old.x - re, old.y - im);
            }
            d.C[i + (int64_t)j * d.ldc] = v;
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tcols));
}

// C (op)= sum over the splits of the FP32 partial tiles, in split order, in FP64.
__global__ void k_zreduce(const ZDesc* __restrict__ descs, int ksplit, int max_m, int max_n,
                          const float* __restrict__ part) {
  const ZDesc d = descs[blockIdx.y];
  if (d.M <= 0 || d.N <= 0 || d.K <= 0) return;
  const int ktd = k_tiles_d(d.K);
  int used = 0;
  for (int y = 0; y < ksplit; ++y) {
    int kb, ke;
    split_range(ktd, ksplit, y, &kb, &ke);
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

inline size_t round256(size_t b) { return (b + 255) / 256 * 256; }

struct Carve {
  Geo g;
  size_t b_off, part_off, total;
};

Carve carve(int mode, int ndesc, int max_m, int max_n, int max_k, int ksplit, bool a_presplit) {
  Carve c;
  c.g.ktc = k_tiles_d(max_k);
  c.g.trb = b_tile_rows(max_n);
  c.g.ksplit = mode == kTN ? std::max(ksplit, 1) : 1;
  c.g.max_m = max_m;
  c.g.max_n = max_n;
  c.g.a_stride = a_presplit ? 0 : round256(a_panel_bytes(max_m, max_k));
  c.g.b_stride = round256((size_t)((2 * max_n + c.g.trb - 1) / c.g.trb) * c.g.ktc * tile_bytes_d(c.g.trb));
  c.b_off = (size_t)ndesc * c.g.a_stride;
  c.part_off = c.b_off + (size_t)ndesc * c.g.b_stride;
  c.total = c.part_off +
            (mode == kTN ? round256((size_t)ndesc * c.g.ksplit * (size_t)max_m * 2 * (size_t)max_n * sizeof(float)) : 0);
  return c;
}

}  // namespace

size_t workspace_bytes(int mode, int ndesc, int max_m, int max_n, int max_k, int ksplit, bool a_presplit) {
  return carve(mode, ndesc, max_m, max_n, max_k, ksplit, a_presplit).total;
}

cudaError_t prepare_zgemm() {
  const int smem = (int)smem_bytes(kTileNMax);
  cudaError_t e = cudaFuncSetAttribute((const void*)k_tc3<kTN>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void*)k_tc3<kNN>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  return e;
}

namespace {
// Split counts worth timing for a kTN product: every count from the accuracy bound's
// minimum up that fills at least 80 % of whole waves of 148 SMs (at most six).
std::vector<int> ksplit_candidates(int ndesc, int max_m, int max_n, int max_k) {
  const int trb = b_tile_rows(max_n);
  const int64_t tiles = (int64_t)((max_m + kTileM - 1) / kTileM) * ((2 * max_n + trb - 1) / trb) * std::max(ndesc, 1);
  const int ktd = k_tiles_d(max_k);
  const int min_split = std::max(1, (ktd + kMaxChain - 1) / kMaxChain);
  const int max_split = std::max(min_split, std::min(64, ktd / 16));
  std::vector<int> out;
  for (int ks = min_split; ks <= max_split && out.size() < 6; ++ks) {
    const int64_t ctas = tiles * ks;
    const int64_t waves = (ctas + kSms - 1) / kSms;
    if ((double)ctas / (double)(waves * kSms) >= 0.8) out.push_back(ks);
  }
  return out;
}

struct TuneEntry {
  int ndesc, m, n, k, chosen;
  std::vector<std::pair<int, float>> timed;  // (split count, ms per product pass)
};
std::mutex g_tune_mu;
std::vector<TuneEntry> g_tuned;
}  // namespace

int tn_ksplit_tuned(int ndesc, int max_m, int max_n, int max_k) {
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (const TuneEntry& e : g_tuned)
      if (e.ndesc == ndesc && e.m == max_m && e.n == max_n && e.k == max_k) return e.chosen;
  }
  const int rule = tn_ksplit(ndesc, max_m, max_n, max_k);
  std::vector<int> cand = ksplit_candidates(ndesc, max_m, max_n, max_k);
  if (std::find(cand.begin(), cand.end(), rule) == cand.end()) cand.push_back(rule);
  TuneEntry entry{ndesc, max_m, max_n, max_k, rule, {}};
  // scratch operands: zeroed panels (their values do not change the time), C and the
  // descriptors; the largest candidate sizes the workspace
  const int kmax = *std::max_element(cand.begin(), cand.end());
  const size_t wb = workspace_bytes(kTN, ndesc, max_m, max_n, max_k, kmax, false);
  const size_t cbytes = (size_t)ndesc * max_m * max_n * sizeof(double2);
  void *work = nullptr, *c = nullptr, *dd = nullptr, *derr = nullptr;
  cudaStream_t s = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  bool ok = cudaMalloc(&work, wb) == cudaSuccess && cudaMalloc(&c, cbytes) == cudaSuccess &&
            cudaMalloc(&dd, sizeof(ZDesc) * ndesc) == cudaSuccess && cudaMalloc(&derr, sizeof(int)) == cudaSuccess &&
            cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreate(&e0) == cudaSuccess && cudaEventCreate(&e1) == cudaSuccess &&
            prepare_zgemm() == cudaSuccess;
  if (ok) {
    std::vector<ZDesc> h((size_t)ndesc);
    for (int z = 0; z < ndesc; ++z)
      h[z] = ZDesc{nullptr, nullptr, static_cast<double2*>(c) + (size_t)z * max_m * max_n, max_k, max_k, max_m,
                   max_m, max_n, max_k, kStore};
    ok = cudaMemsetAsync(work, 0, wb, s) == cudaSuccess && cudaMemsetAsync(derr, 0, sizeof(int), s) == cudaSuccess &&
         cudaMemcpyAsync(dd, h.data(), sizeof(ZDesc) * ndesc, cudaMemcpyHostToDevice, s) == cudaSuccess;
  }
  float best = 0.0f;
  for (size_t i = 0; ok && i < cand.size(); ++i) {
    const Carve cv = carve(kTN, ndesc, max_m, max_n, max_k, cand[i], false);
    unsigned char* w = static_cast<unsigned char*>(work);
    const unsigned tiles = (unsigned)(((max_m + kTileM - 1) / kTileM) * ((2 * max_n + cv.g.trb - 1) / cv.g.trb));
    const int64_t total = (int64_t)max_m * max_n;
    const unsigned rblocks = (unsigned)std::min<int64_t>((total + 255) / 256, 1024);
    float t = 0.0f;
    for (int rep = 0; rep < 3 && ok; ++rep) {  // the first launch warms, the best of two counts
      ok = cudaEventRecord(e0, s) == cudaSuccess;
      k_tc3<kTN><<<dim3(tiles, (unsigned)cv.g.ksplit, (unsigned)ndesc), kThreads, smem_bytes(cv.g.trb), s>>>(
          static_cast<const ZDesc*>(dd), cv.g, w, w + cv.b_off, reinterpret_cast<float*>(w + cv.part_off),
          static_cast<int*>(derr));
      k_zreduce<<<dim3(rblocks, (unsigned)ndesc), 256, 0, s>>>(static_cast<const ZDesc*>(dd), cv.g.ksplit, max_m,
                                                               max_n, reinterpret_cast<float*>(w + cv.part_off));
      ok = ok && cudaEventRecord(e1, s) == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess;
      float ms = 0.0f;
      if (ok) ok = cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess;
      if (rep == 1 || (rep == 2 && ms < t)) t = ms;
    }
    if (!ok) break;
    entry.timed.push_back({cand[i], t});
    if (i == 0 || t < best) {
      best = t;
      entry.chosen = cand[i];
    }
  }
  int herr = 0;
  if (ok && cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess && herr) ok = false;
  if (!ok) entry.chosen = rule;  // a failed measurement keeps the rule's count
  cudaGetLastError();
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (s) cudaStreamDestroy(s);
  cudaFree(work);
  cudaFree(c);
  cudaFree(dd);
  cudaFree(derr);
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tuned.push_back(entry);
  return entry.chosen;
}

std::string tuning_report() {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  std::string out = "[";
  for (size_t i = 0; i < g_tuned.size(); ++i) {
    const TuneEntry& e = g_tuned[i];
    char head[160];
    std::snprintf(head, sizeof head, "%s{\"product\": \"A^H B\", \"ndesc\": %d, \"m\": %d, \"n\": %d, \"k\": %d, "
                  "\"ksplit\": %d, \"timed_ms\": {", i ? ", " : "", e.ndesc, e.m, e.n, e.k, e.chosen);
    out += head;
    for (size_t j = 0; j < e.timed.size(); ++j) {
      char item[48];
      std::snprintf(item, sizeof item, "%s\"%d\": %.4f", j ? ", " : "", e.timed[j].first, e.timed[j].second);
      out += item;
    }
    out += "}}";
  }
  return out + "]";
}

int tn_ksplit(int ndesc, int max_m, int max_n, int max_k) {
  const int trb = b_tile_rows(max_n);
  const int64_t tiles = (int64_t)((max_m + kTileM - 1) / kTileM) * ((2 * max_n + trb - 1) / trb) * std::max(ndesc, 1);
  const int ktd = k_tiles_d(max_k);
  // The FP32 accumulation in tensor memory adds an error that grows with the number of
  // K tiles a CTA accumulates: at most kMaxChain tiles (4,096 complex K) per split.
  const int min_split = std::max(1, (ktd + kMaxChain - 1) / kMaxChain);
  const int max_split = std::max(min_split, std::min(64, ktd / 16));  // at least 16 K tiles each
  int best = min_split;
  double best_eff = 0.0;
  for (int ks = min_split; ks <= max_split; ++ks) {
    const int64_t ctas = tiles * ks;
    const int64_t waves = (ctas + kSms - 1) / kSms;
    const double eff = (double)ctas / (double)(waves * kSms);
    if (eff >= 0.9) return ks;
    if (eff > best_eff + 1e-9) {
      best_eff = eff;
      best = ks;
    }
  }
  return best;
}

int launch_zgemm(int mode, const ZDesc* d_desc, int ndesc, int max_m, int max_n, int max_k, int ksplit,
                 bool a_presplit, void* work, int* err, cudaStream_t s) {
  if (ndesc == 0 || max_m <= 0 || max_n <= 0 || max_k <= 0) return 0;
  const Carve c = carve(mode, ndesc, max_m, max_n, max_k, ksplit, a_presplit);
  unsigned char* w = static_cast<unsigned char*>(work);
  int launches = 0;
  if (!a_presplit) {
    const unsigned rt = (unsigned)((max_m + kTileM - 1) / kTileM);
    const unsigned gx = split_blocks((int64_t)c.g.ktc * kTileM);
    k_split_desc<<<dim3(gx, rt, (unsigned)ndesc), 256, 0, s>>>(d_desc, mode, 0, kTileM, c.g.ktc, c.g.a_stride, w);
    ++launches;
  }
  {
    const unsigned rt = (unsigned)((2 * max_n + c.g.trb - 1) / c.g.trb);
    const unsigned gx = split_blocks((int64_t)c.g.ktc * (c.g.trb / 2));
    k_split_desc<<<dim3(gx, rt, (unsigned)ndesc), 256, 0, s>>>(d_desc, mode, 1, c.g.trb, c.g.ktc, c.g.b_stride,
                                                               w + c.b_off);
    ++launches;
  }
  const unsigned tiles = (unsigned)(((max_m + kTileM - 1) / kTileM) * ((2 * max_n + c.g.trb - 1) / c.g.trb));
  const size_t smem = smem_bytes(c.g.trb);
  float* part = reinterpret_cast<float*>(w + c.part_off);
  if (mode == kTN) {
    k_tc3<kTN><<<dim3(tiles, (unsigned)c.g.ksplit, (unsigned)ndesc), kThreads, smem, s>>>(d_desc, c.g, w, w + c.b_off,
                                                                                          part, err);
    const int64_t total = (int64_t)max_m * max_n;
    const unsigned blocks = (unsigned)std::min<int64_t>((total + 255) / 256, 1024);
    k_zreduce<<<dim3(blocks, (unsigned)ndesc), 256, 0, s>>>(d_desc, c.g.ksplit, max_m, max_n, part);
    return launches + 2;
  }
  k_tc3<kNN><<<dim3(tiles, 1, (unsigned)ndesc), kThreads, smem, s>>>(d_desc, c.g, w, w + c.b_off, nullptr, err);
  return launches + 1;
}

cudaError_t split_a(int mode, const double2* A, int64_t lda, int M, int K, unsigned char* panel, cudaStream_t s) {
  if (M <= 0 || K <= 0) return cudaSuccess;
  SplitArgs a;
  a.X = A;
  a.K = K;
  a.cols = M;
  a.nvar = 1;
  a.var = kVarA;
  a.sk = mode == kTN ? 1 : lda;
  a.sj = mode == kTN ? lda : 1;
  a.R = kTileM;
  a.ktc = k_tiles_d(K);
  a.panel = panel;
  const unsigned rt = (unsigned)((M + kTileM - 1) / kTileM);
  k_split_args<<<dim3(split_blocks((int64_t)a.ktc * kTileM), rt), 256, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace tc
}  // namespace bg

// ------------------------------------------------------------------ C ABI
#include <cstring>
#include <string>

#include "op_internal.h"

using namespace bg;

extern "C" int bg_autotune_report(char* buf, int64_t capacity) {
  const std::string r = tc::tuning_report();
  if (!buf || capacity <= 0) return (int)r.size() + 1;
  const size_t n = std::min<size_t>(r.size(), (size_t)capacity - 1);
  std::memcpy(buf, r.data(), n);
  buf[n] = 0;
  return (int)r.size() + 1;
}

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
  void* work = nullptr;
  const size_t wb = tc::workspace_bytes(mode, 1, (int)m, (int)n, (int)k, ks, false);
  e = cudaMalloc(&dd, sizeof(tc::ZDesc));
  if (e == cudaSuccess) e = cudaMalloc(&derr, sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&work, wb);
  int herr = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(dd, &d, sizeof d, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(derr, 0, sizeof(int), s);
  if (e == cudaSuccess) {
    tc::launch_zgemm(mode, dd, 1, (int)m, (int)n, (int)k, ks, false, work, derr, s);
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
