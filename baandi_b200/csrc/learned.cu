// Learned preconditioner: training samples, the loss and its gradient, the Adam step
// (BF16 weights, FP32 accumulation), and the context's inference parameters.  The network
// and its inputs are defined in learned.cuh; BG_PRECOND_LEARNED (correction_column) runs
// its inference.
//
// A training sample is one (row g, band j) of a Davidson state: inputs f_gj, the TPA
// factor b_g = -tpa(t_g, s_j), a_g = |r_g|^2 and z_g = conj(r_g) e_g, where e_j is the
// ideal correction of band j (the part of the Ritz vector outside the exact eigenspace).
// The correction c = p r with p = b exp(clamp(m(f))) is scored per band by its squared
// cosine with e: with A_j = sum_g p_g z_g, B_j = sum_g p_g^2 a_g and E_j = |e_j|^2,
//   loss = (1 / ncols) sum_j (1 - |A_j|^2 / (B_j E_j)),
// which ignores the scale of each correction, as the Davidson does.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "blas_dev.cuh"
#include "learned.cuh"
#include "op_internal.h"

namespace bg {
namespace {

using learned::kHid;
using learned::kIn;
using learned::kParams;

// One 256-thread block per band column j: the column's samples at j * rows.
template <class D>
__global__ void __launch_bounds__(256) k_learned_samples(const D* __restrict__ X, const D* __restrict__ HX,
                                                          const D* __restrict__ Et, const double* __restrict__ kin,
                                                          const double* __restrict__ lam, int64_t rows, int col0,
                                                          float* __restrict__ feats, float* __restrict__ base,
                                                          float* __restrict__ a, float2* __restrict__ z,
                                                          int* __restrict__ col, double* __restrict__ ecol) {
  __shared__ double red[256];
  const int j = blockIdx.x;
  const D* x = X + j * rows;
  const D* hx = HX + j * rows;
  const D* e = Et + j * rows;
  const double lj = lam[j];
  double w = 0.0, wt = 0.0, q = 0.0, ee = 0.0;
  for (int64_t r = threadIdx.x; r < rows; r += blockDim.x) {
    const double xa = Arith<D>::norm2(x[r]);
    w += xa;
    wt += xa * kin[r];
    q += Arith<D>::norm2(Arith<D>::add(hx[r], Arith<D>::scale(-lj, x[r])));
    ee += Arith<D>::norm2(e[r]);
  }
  w = block_sum256(w, red);
  wt = block_sum256(wt, red);
  q = block_sum256(q, red);
  ee = block_sum256(ee, red);
  const double s = fmax(wt / w, 0.1);
  const double rms = sqrt(q / (double)rows);
  const int64_t o = (int64_t)j * rows;  // this column's samples (arrays offset by the caller)
  for (int64_t r = threadIdx.x; r < rows; r += blockDim.x) {
    const D res = Arith<D>::add(hx[r], Arith<D>::scale(-lj, x[r]));
    const double ra = Arith<D>::norm2(res);
    float f[kIn];
    learned::features(kin[r], s, lj, rms > 0.0 ? sqrt(ra) / rms : 1.0, f);
#pragma unroll
    for (int k = 0; k < kIn; ++k) feats[(o + r) * kIn + k] = f[k];
    base[o + r] = (float)(-tpa_weight(kin[r], s));
    a[o + r] = (float)ra;
    double zr, zi;
    if constexpr (sizeof(D) == sizeof(double)) {
      zr = (double)res * (double)e[r];
      zi = 0.0;
    } else {
      const double2 rr = reinterpret_cast<const double2&>(res);
      const double2 ev = reinterpret_cast<const double2&>(e[r]);
      zr = rr.x * ev.x + rr.y * ev.y;  // conj(r) e
      zi = rr.x * ev.y - rr.y * ev.x;
    }
    z[o + r] = make_float2((float)zr, (float)zi);
    col[o + r] = col0 + j;
  }
  if (threadIdx.x == 0) ecol[col0 + j] = ee;
}

// Forward over the samples: p_n and the column sums A_j (complex) and B_j.
__global__ void __launch_bounds__(128) k_learned_forward(const float* __restrict__ feats, const float* __restrict__ base,
                                                          const float* __restrict__ a, const float2* __restrict__ z,
                                                          const int* __restrict__ col, int64_t n,
                                                          const __nv_bfloat16* __restrict__ net, float* __restrict__ p,
                                                          double* __restrict__ colsum) {
  __shared__ float w[kParams];
  learned::load_params(net, w);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float f[kIn];
#pragma unroll
    for (int k = 0; k < kIn; ++k) f[k] = feats[i * kIn + k];
    const float m = learned::forward(w, f);
    const float pv = base[i] * expf(fminf(fmaxf(m, -learned::kClamp), learned::kClamp));
    p[i] = pv;
    const int c = col[i];
    atomicAdd(colsum + 3 * c + 0, (double)pv * z[i].x);
    atomicAdd(colsum + 3 * c + 1, (double)pv * z[i].y);
    atomicAdd(colsum + 3 * c + 2, (double)pv * pv * a[i]);
  }
}

// loss and the per-column coefficients of dloss/dp_n = -Re(conj(cA_j) z_n) + cB_j p_n a_n:
// cA = 2 A / (B E ncols), cB = 2 |A|^2 / (B^2 E ncols) (coef[3 j ..]); columns with B or E
// zero add nothing.  One block of 256 threads; the loss sum runs in a fixed order.
__global__ void __launch_bounds__(256) k_learned_loss(const double* __restrict__ colsum, const double* __restrict__ ecol,
                                                      int ncols, double* __restrict__ coef, double* __restrict__ loss) {
  __shared__ double red[256];
  double l = 0.0;
  for (int j = threadIdx.x; j < ncols; j += blockDim.x) {
    const double ar = colsum[3 * j], ai = colsum[3 * j + 1], b = colsum[3 * j + 2], e = ecol[j];
    double ca_r = 0.0, ca_i = 0.0, cb = 0.0;
    if (b > 0.0 && e > 0.0) {
      const double a2 = ar * ar + ai * ai;
      l += 1.0 - a2 / (b * e);
      ca_r = 2.0 * ar / (b * e * ncols);
      ca_i = 2.0 * ai / (b * e * ncols);
      cb = 2.0 * a2 / (b * b * e * ncols);
    }
    coef[3 * j] = ca_r;
    coef[3 * j + 1] = ca_i;
    coef[3 * j + 2] = cb;
  }
  l = block_sum256(l, red);
  if (threadIdx.x == 0) *loss = l / ncols;
}

// Backward: tiles of 64 samples (one per thread) through the network, then each thread
// adds the tile's gradient of its own parameters (t, t + 64, ...) into registers; one
// atomic add per parameter per block at the end.
constexpr int kTile = 64;
constexpr int kLd = kHid + 1;  // padded rows: thread s reads row s without bank conflicts
constexpr int kOwn = (kParams + kTile - 1) / kTile;
constexpr size_t kBwdSmem =
    sizeof(float) * ((size_t)kParams + 4 * (size_t)kTile * kLd + (size_t)kTile * kIn + kTile);

__global__ void __launch_bounds__(kTile) k_learned_backward(const float* __restrict__ feats,
                                                            const float* __restrict__ a, const float2* __restrict__ z,
                                                            const int* __restrict__ col, const float* __restrict__ p,
                                                            int64_t n, const __nv_bfloat16* __restrict__ net,
                                                            const double* __restrict__ coef, float* __restrict__ grad) {
  extern __shared__ float sm[];
  float* w = sm;
  float* H1 = w + kParams;        // [s][i] gelu(pre1)
  float* D1 = H1 + kTile * kLd;   // [s][i] gelu'(pre1), then delta1
  float* H2 = D1 + kTile * kLd;   // [s][o] gelu(pre2)
  float* D2 = H2 + kTile * kLd;   // [s][o] delta2
  float* F = D2 + kTile * kLd;    // [s][k] inputs
  float* DO = F + kTile * kIn;    // [s] dloss/dm
  learned::load_params(net, w);
  float acc[kOwn];
#pragma unroll
  for (int q = 0; q < kOwn; ++q) acc[q] = 0.0f;
  const int s = threadIdx.x;
  const int64_t ntiles = (n + kTile - 1) / kTile;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t i = tile * kTile + s;
    const bool live = i < n;
    float* h1 = H1 + s * kLd;
    float* d1 = D1 + s * kLd;
    float* h2 = H2 + s * kLd;
    float* d2 = D2 + s * kLd;
    float f[kIn];
#pragma unroll
    for (int k = 0; k < kIn; ++k) {
      f[k] = live ? feats[i * kIn + k] : 0.0f;
      F[s * kIn + k] = f[k];
    }
    for (int u = 0; u < kHid; ++u) {
      float pre = w[learned::oB1 + u];
#pragma unroll
      for (int k = 0; k < kIn; ++k) pre = fmaf(w[learned::oW1 + u * kIn + k], f[k], pre);
      h1[u] = learned::gelu(pre);
      d1[u] = learned::gelu_grad(pre);
    }
    float m = w[learned::oB3];
    for (int o = 0; o < kHid; ++o) {
      float pre = w[learned::oB2 + o];
#pragma unroll 8
      for (int u = 0; u < kHid; ++u) pre = fmaf(w[learned::oW2 + o * kHid + u], h1[u], pre);
      h2[o] = learned::gelu(pre);
      d2[o] = learned::gelu_grad(pre);  // delta2 once dm is known
      m = fmaf(w[learned::oW3 + o], h2[o], m);
    }
    float dm = 0.0f;
    if (live && fabsf(m) < learned::kClamp) {
      const int c = col[i];
      const double pv = p[i];
      const double dp = -(coef[3 * c] * z[i].x + coef[3 * c + 1] * z[i].y) + coef[3 * c + 2] * pv * a[i];
      dm = (float)(dp * pv);  // dp/dm = p inside the clamp
    }
    DO[s] = dm;
    for (int o = 0; o < kHid; ++o) d2[o] *= dm * w[learned::oW3 + o];
    for (int u = 0; u < kHid; ++u) {
      float t = 0.0f;
#pragma unroll 8
      for (int o = 0; o < kHid; ++o) t = fmaf(w[learned::oW2 + o * kHid + u], d2[o], t);
      d1[u] *= t;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kOwn; ++q) {
      const int e = s + q * kTile;
      if (e >= kParams) break;
      float g = 0.0f;
      if (e < learned::oB1) {  // W1[u][k]
        const int u = e / kIn, k = e - u * kIn;
        for (int t = 0; t < kTile; ++t) g = fmaf(D1[t * kLd + u], F[t * kIn + k], g);
      } else if (e < learned::oW2) {
        const int u = e - learned::oB1;
        for (int t = 0; t < kTile; ++t) g += D1[t * kLd + u];
      } else if (e < learned::oB2) {  // W2[o][u]
        const int o = (e - learned::oW2) / kHid, u = (e - learned::oW2) - o * kHid;
        for (int t = 0; t < kTile; ++t) g = fmaf(D2[t * kLd + o], H1[t * kLd + u], g);
      } else if (e < learned::oW3) {
        const int o = e - learned::oB2;
        for (int t = 0; t < kTile; ++t) g += D2[t * kLd + o];
      } else if (e < learned::oB3) {
        const int o = e - learned::oW3;
        for (int t = 0; t < kTile; ++t) g = fmaf(DO[t], H2[t * kLd + o], g);
      } else {
        for (int t = 0; t < kTile; ++t) g += DO[t];
      }
      acc[q] += g;
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < kOwn; ++q) {
    const int e = s + q * kTile;
    if (e < kParams) atomicAdd(grad + e, acc[q]);
  }
}

// Adam (beta1 0.9, beta2 0.999, eps 1e-8, bias-corrected) on the FP32 master copy; the
// BF16 copy the network runs with is rounded from it.
__global__ void k_learned_adam(float* __restrict__ master, float* __restrict__ m1, float* __restrict__ m2,
                               const float* __restrict__ grad, __nv_bfloat16* __restrict__ net, int step, float lr) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= kParams) return;
  const float g = grad[e];
  const float a = 0.9f * m1[e] + 0.1f * g;
  const float b = 0.999f * m2[e] + 0.001f * g * g;
  m1[e] = a;
  m2[e] = b;
  const float ah = a / (1.0f - powf(0.9f, (float)step));
  const float bh = b / (1.0f - powf(0.999f, (float)step));
  const float v = master[e] - lr * ah / (sqrtf(bh) + 1e-8f);
  master[e] = v;
  net[e] = __float2bfloat16_rn(v);
}

// Round to nearest even BF16 (NaN stays NaN).
uint16_t to_bf16(float v) {
  uint32_t u;
  std::memcpy(&u, &v, 4);
  if ((u & 0x7f800000u) == 0x7f800000u && (u & 0x007fffffu)) return (uint16_t)((u >> 16) | 0x40u);
  u += 0x7fffu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}

int lfail(bg_ctx* ctx, int code, const char* msg) {
  if (ctx) ctx->error = msg;
  return code;
}

int lcheck(bg_ctx* ctx, const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    if (ctx) ctx->error = std::string(what) + ": " + cudaGetErrorString(e);
    return BG_EDEVICE;
  }
  return BG_OK;
}

}  // namespace
}  // namespace bg

using namespace bg;

extern "C" int bg_learned_set(bg_ctx* ctx, const float* params) {
  if (!ctx || !params) return lfail(ctx, BG_EINVAL, "null argument");
  std::vector<uint16_t> h(kParams);
  for (int i = 0; i < kParams; ++i) {
    if (!std::isfinite(params[i])) return lfail(ctx, BG_ENONFINITE, "learned preconditioner parameters not finite");
    h[i] = to_bf16(params[i]);
  }
  {
    const cudaError_t de = cudaSetDevice(ctx->device);
    if (de != cudaSuccess) return lfail(ctx, BG_EDEVICE, cudaGetErrorString(de));
  }
  if (!ctx->learned && cudaMalloc(&ctx->learned, sizeof(uint16_t) * kParams) != cudaSuccess) {
    ctx->learned = nullptr;
    return lfail(ctx, BG_ENOMEM, "learned preconditioner parameters");
  }
  if (cudaMemcpy(ctx->learned, h.data(), sizeof(uint16_t) * kParams, cudaMemcpyHostToDevice) != cudaSuccess)
    return lfail(ctx, BG_EDEVICE, "learned preconditioner upload");
  return BG_OK;
}

extern "C" int bg_learned_clear(bg_ctx* ctx) {
  if (!ctx) return BG_EINVAL;
  if (ctx->learned) cudaFree(ctx->learned);
  ctx->learned = nullptr;
  return BG_OK;
}

extern "C" int bg_learned_samples_build(bg_ctx* ctx, int64_t rows, int32_t cols, int32_t is_complex, const double* x,
                                        const double* hx, const double* target, const double* kinetic,
                                        const double* lambda, int32_t col0, int64_t at, const bg_learned_samples* out,
                                        void* stream) {
  if (!ctx || !x || !hx || !target || !kinetic || !lambda || !out || rows <= 0 || cols <= 0 || col0 < 0 || at < 0)
    return lfail(ctx, BG_EINVAL, "learned samples: arguments");
  if (col0 + (int64_t)cols > out->ncols || at + (int64_t)cols * rows > out->n)
    return lfail(ctx, BG_EINVAL, "learned samples: output too small");
  {
    const cudaError_t de = cudaSetDevice(ctx->device);
    if (de != cudaSuccess) return lfail(ctx, BG_EDEVICE, cudaGetErrorString(de));
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  float* feats = out->feats + at * kIn;
  float2* z = reinterpret_cast<float2*>(out->z) + at;
  if (is_complex)
    k_learned_samples<double2><<<cols, 256, 0, s>>>(
        reinterpret_cast<const double2*>(x), reinterpret_cast<const double2*>(hx),
        reinterpret_cast<const double2*>(target), kinetic, lambda, rows, col0, feats, out->base + at, out->a + at, z,
        out->col + at, out->ecol);
  else
    k_learned_samples<double><<<cols, 256, 0, s>>>(x, hx, target, kinetic, lambda, rows, col0, feats, out->base + at,
                                                   out->a + at, z, out->col + at, out->ecol);
  return lcheck(ctx, "learned samples");
}

extern "C" int bg_learned_loss_grad(bg_ctx* ctx, const bg_learned_samples* smp, const uint16_t* net, float* grad,
                                    double* work, double* loss, void* stream) {
  if (!ctx || !smp || !net || !grad || !work || smp->n <= 0 || smp->ncols <= 0)
    return lfail(ctx, BG_EINVAL, "learned loss: arguments");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int nc = smp->ncols;
  double* colsum = work;
  double* coef = work + 3 * (size_t)nc;
  double* dloss = work + 6 * (size_t)nc;
  float* p = reinterpret_cast<float*>(work + 6 * (size_t)nc + 1);
  const auto* bnet = reinterpret_cast<const __nv_bfloat16*>(net);
  {
    const cudaError_t de = cudaSetDevice(ctx->device);
    if (de != cudaSuccess) return lfail(ctx, BG_EDEVICE, cudaGetErrorString(de));
  }
  // per device and cheap: set on every call
  if (cudaFuncSetAttribute(k_learned_backward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBwdSmem) !=
      cudaSuccess)
    return lcheck(ctx, "learned backward shared memory");
  cudaMemsetAsync(colsum, 0, sizeof(double) * 3 * (size_t)nc, s);
  cudaMemsetAsync(grad, 0, sizeof(float) * kParams, s);
  const int64_t fb = std::min<int64_t>((smp->n + 127) / 128, 148 * 8);
  k_learned_forward<<<(unsigned)fb, 128, 0, s>>>(smp->feats, smp->base, smp->a, reinterpret_cast<const float2*>(smp->z),
                                                 smp->col, smp->n, bnet, p, colsum);
  k_learned_loss<<<1, 256, 0, s>>>(colsum, smp->ecol, nc, coef, dloss);
  const int64_t bb = std::min<int64_t>((smp->n + kTile - 1) / kTile, 148 * 2);
  k_learned_backward<<<(unsigned)bb, kTile, kBwdSmem, s>>>(smp->feats, smp->a, reinterpret_cast<const float2*>(smp->z),
                                                          smp->col, p, smp->n, bnet, coef, grad);
  int rc = lcheck(ctx, "learned loss/grad");
  if (rc) return rc;
  if (loss) {
    if (cudaMemcpyAsync(loss, dloss, sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      return lfail(ctx, BG_EDEVICE, "learned loss read");
  }
  return BG_OK;
}

extern "C" int bg_learned_adam(bg_ctx* ctx, float* master, float* m1, float* m2, const float* grad, uint16_t* net,
                               int32_t step, float lr, void* stream) {
  if (!ctx || !master || !m1 || !m2 || !grad || !net || step < 1 || !(lr > 0.0f))
    return lfail(ctx, BG_EINVAL, "learned adam: arguments");
  {
    const cudaError_t de = cudaSetDevice(ctx->device);
    if (de != cudaSuccess) return lfail(ctx, BG_EDEVICE, cudaGetErrorString(de));
  }
  k_learned_adam<<<(kParams + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      master, m1, m2, grad, reinterpret_cast<__nv_bfloat16*>(net), step, lr);
  return lcheck(ctx, "learned adam");
}
