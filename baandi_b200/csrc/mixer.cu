// Density mixing of the SCF map on the GPU: the reference's unnormalised
// difference-history Anderson (Broyden) update with its Hartree metric, FP64.
//
// Reference: crates/dft-engine/src/refscf/broyden.rs:96-123 (screening), 319-435
// (update); crates/dft-engine/src/refscf/metric.rs:22-47 (weights 8 pi Omega / G^2 on
// smooth G != 0), 175-190 (compensated sums).  The history ring, slot and occupancy
// depend only on the iteration count, so they are tracked on the host; every vector
// operation and the small symmetric solve run on the device:
//   k_mix_diff   dF[slot] = F_prev - F, dx[slot] = x_prev - x, then x_prev, F_prev
//   k_mix_forms  one block per Gram entry <dF_i, dF_j> and right-hand side <dF_i, F>,
//                Neumaier-compensated per thread and combined in a fixed tree
//   k_mix_solve  A = Q diag(lambda) Q^T by cyclic Jacobi (p <= 25), the rank test
//                lambda_min <= p eps lambda_max, gamma = Q diag(1/lambda) Q^T b
//   k_mix_apply  next = x~ + beta s F~ on smooth G (x~ = x - gamma.dx, F~ = F - gamma.dF),
//                next = x + beta F elsewhere; F~ kept as the reduced residual
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <memory>
#include <string>
#include <vector>

#include "op_internal.h"

namespace bg {
namespace {

constexpr int kMaxHistory = 25;
constexpr int kMaxForms = kMaxHistory * (kMaxHistory + 1) / 2 + kMaxHistory;
constexpr int kMixThreads = 256;
constexpr double kPi = 3.14159265358979323846;
constexpr double kEps = 2.220446049250313e-16;

struct Neu {
  double s, c;
};
__device__ __forceinline__ void neu_add(Neu& a, double v) {
  const double t = a.s + v;
  a.c += fabs(a.s) >= fabs(v) ? (a.s - t) + v : (v - t) + a.s;
  a.s = t;
}

__global__ void k_mix_diff(const double2* __restrict__ x, const double2* __restrict__ f, double2* prev_x,
                           double2* prev_f, double2* __restrict__ dx, double2* __restrict__ df, int64_t n, int have_slot) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
    const double2 xv = x[j], fv = f[j];
    if (have_slot) {
      const double2 px = prev_x[j], pf = prev_f[j];
      df[j] = make_double2(pf.x - fv.x, pf.y - fv.y);
      dx[j] = make_double2(px.x - xv.x, px.y - xv.y);
    }
    prev_x[j] = xv;
    prev_f[j] = fv;
  }
}

// forms[q] for q < p(p+1)/2: <dF_i, dF_j> (i >= j, row-major lower triangle);
// forms[p(p+1)/2 + i] = <dF_i, F>.  One block per form.
__global__ void __launch_bounds__(kMixThreads) k_mix_forms(const double2* __restrict__ df, int64_t n, int p,
                                                           const double2* __restrict__ f,
                                                           const double* __restrict__ w, double* __restrict__ forms) {
  const int q = blockIdx.x;
  const int tri = p * (p + 1) / 2;
  const double2* a;
  const double2* b;
  if (q < tri) {
    int i = 0;
    while ((i + 1) * (i + 2) / 2 <= q) ++i;
    const int j = q - i * (i + 1) / 2;
    a = df + (int64_t)i * n;
    b = df + (int64_t)j * n;
  } else {
    a = df + (int64_t)(q - tri) * n;
    b = f;
  }
  Neu acc{0.0, 0.0};
  for (int64_t t = threadIdx.x; t < n; t += blockDim.x) {
    const double2 u = a[t], v = b[t];
    neu_add(acc, w[t] * (u.x * v.x + u.y * v.y));
  }
  __shared__ double ss[kMixThreads], sc[kMixThreads];
  ss[threadIdx.x] = acc.s;
  sc[threadIdx.x] = acc.c;
  __syncthreads();
  for (int st = kMixThreads / 2; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st) {
      Neu m{ss[threadIdx.x], sc[threadIdx.x] + sc[threadIdx.x + st]};
      neu_add(m, ss[threadIdx.x + st]);
      ss[threadIdx.x] = m.s;
      sc[threadIdx.x] = m.c;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) forms[q] = ss[0] + sc[0];
}

// One thread: Jacobi eigen-decomposition of the p x p Gram, rank test, gamma.
// out[0] = status (0 ok, 1 singular, 2 non-finite), out[1] = lambda_min,
// out[2] = lambda_max, out[3] = condition.
__global__ void k_mix_solve(const double* __restrict__ forms, int p, double* __restrict__ gamma,
                            double* __restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double A[kMaxHistory][kMaxHistory], Q[kMaxHistory][kMaxHistory];
  int idx = 0;
  bool finite = true;
  for (int i = 0; i < p; ++i)
    for (int j = 0; j <= i; ++j) {
      const double v = forms[idx++];
      finite &= isfinite(v);
      A[i][j] = A[j][i] = v;
    }
  const double* b = forms + idx;
  for (int i = 0; i < p; ++i) {
    finite &= isfinite(b[i]);
    for (int j = 0; j < p; ++j) Q[i][j] = i == j ? 1.0 : 0.0;
  }
  if (!finite) {
    out[0] = 2.0;
    return;
  }
  double norm = 0.0;
  for (int i = 0; i < p; ++i)
    for (int j = 0; j < p; ++j) norm += A[i][j] * A[i][j];
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0.0;
    for (int i = 0; i < p; ++i)
      for (int j = 0; j < i; ++j) off += A[i][j] * A[i][j];
    if (off <= 1e-32 * norm) break;
    for (int r = 0; r < p; ++r)
      for (int s = r + 1; s < p; ++s) {
        const double ars = A[r][s];
        if (ars == 0.0) continue;
        const double theta = (A[s][s] - A[r][r]) / (2.0 * ars);
        const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0), sn = t * c;
        for (int k = 0; k < p; ++k) {
          const double akr = A[k][r], aks = A[k][s];
          A[k][r] = c * akr - sn * aks;
          A[k][s] = sn * akr + c * aks;
        }
        for (int k = 0; k < p; ++k) {
          const double ark = A[r][k], ask = A[s][k];
          A[r][k] = c * ark - sn * ask;
          A[s][k] = sn * ark + c * ask;
        }
        for (int k = 0; k < p; ++k) {
          const double qkr = Q[k][r], qks = Q[k][s];
          Q[k][r] = c * qkr - sn * qks;
          Q[k][s] = sn * qkr + c * qks;
        }
      }
  }
  double lo = A[0][0], hi = A[0][0];
  for (int i = 1; i < p; ++i) {
    lo = fmin(lo, A[i][i]);
    hi = fmax(hi, A[i][i]);
  }
  const double cond = lo > 0.0 ? hi / lo : INFINITY;
  out[1] = lo;
  out[2] = hi;
  out[3] = cond;
  if (lo <= p * kEps * hi || !isfinite(cond)) {
    out[0] = 1.0;
    return;
  }
  double g[kMaxHistory];
  for (int i = 0; i < p; ++i) g[i] = 0.0;
  for (int j = 0; j < p; ++j) {
    double proj = 0.0;
    for (int i = 0; i < p; ++i) proj += Q[i][j] * b[i];
    for (int i = 0; i < p; ++i) g[i] += Q[i][j] * (proj / A[j][j]);
  }
  for (int i = 0; i < p; ++i) gamma[i] = g[i];
  out[0] = 0.0;
}

__global__ void k_mix_apply(const double2* __restrict__ x, const double2* __restrict__ f,
                            const double2* __restrict__ dx, const double2* __restrict__ df, int64_t n, int p,
                            const double* __restrict__ gamma, const int* __restrict__ smooth,
                            const double* __restrict__ screening, double beta, double2* __restrict__ next,
                            double2* __restrict__ reduced, int* err) {
  __shared__ double g[kMaxHistory];
  if ((int)threadIdx.x < p) g[threadIdx.x] = gamma[threadIdx.x];
  __syncthreads();
  bool bad = false;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
    double2 xx = x[j], ff = f[j];
    if (smooth[j]) {
      for (int i = 0; i < p; ++i) {
        const double2 a = dx[(int64_t)i * n + j], c = df[(int64_t)i * n + j];
        xx.x -= g[i] * a.x;
        xx.y -= g[i] * a.y;
        ff.x -= g[i] * c.x;
        ff.y -= g[i] * c.y;
      }
      reduced[j] = ff;
      ff.x *= screening[j];
      ff.y *= screening[j];
    } else {
      reduced[j] = ff;
    }
    const double2 v = make_double2(xx.x + beta * ff.x, xx.y + beta * ff.y);
    bad |= !(isfinite(v.x) && isfinite(v.y));
    next[j] = v;
  }
  if (bad) atomicOr(err, 1);
}

}  // namespace
}  // namespace bg

using namespace bg;

struct bg_mixer {
  bg_ctx* ctx = nullptr;
  int64_t n = 0;
  double beta = 0.7;
  int history = 8;
  int iteration = 0;
  bool failed = false;
  int occupancy = 0;
  double2 *prev_x = nullptr, *prev_f = nullptr, *dx = nullptr, *df = nullptr, *reduced = nullptr;
  double2 *sx = nullptr, *sf = nullptr, *snext = nullptr;  // host-pointer staging
  double *w = nullptr, *screening = nullptr, *forms = nullptr, *gamma = nullptr, *out = nullptr;
  int* smooth = nullptr;
  int* err = nullptr;
  double* host_out = nullptr;  // pinned: out[4], err, gamma[25]
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::vector<std::unique_ptr<DevBuf>> bufs;
};

namespace {
int malloc_into(bg_mixer* m, size_t bytes, void** p) {
  auto b = std::make_unique<DevBuf>();
  b->bytes = std::max<size_t>(bytes, 16);
  cudaError_t e = cudaMalloc(&b->p, b->bytes);
  if (e != cudaSuccess) return fail(m->ctx, BG_ENOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  cudaMemset(b->p, 0, b->bytes);
  *p = b->p;
  m->bufs.push_back(std::move(b));
  return BG_OK;
}
template <class P>
int dalloc(bg_mixer* m, P** p, size_t count) {
  void* v = nullptr;
  int rc = malloc_into(m, count * sizeof(P), &v);
  *p = static_cast<P*>(v);
  return rc;
}
unsigned grid_for(int64_t n) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 4 * 148)); }
}  // namespace

extern "C" {

int bg_mixer_create(bg_ctx* ctx, const bg_mixer_profile* profile, int64_t n, const double* g2, const int32_t* smooth,
                    double volume, double electrons, double metric_volume, bg_mixer** out) {
  if (!ctx || !profile || !g2 || !smooth || !out) return fail(ctx, BG_EINVAL, "null argument");
  const bg_mixer_profile p = *profile;
  if (!std::isfinite(p.beta) || !(p.beta > 0.0 && p.beta <= 1.0))
    return fail(ctx, BG_EINVAL, "beta must be finite and in (0,1]");
  if (p.history < 1 || p.history > kMaxHistory) return fail(ctx, BG_EINVAL, "history must be in 1..=25");
  if (n < 1 || !std::isfinite(volume) || volume <= 0.0 || !std::isfinite(electrons) || electrons <= 0.0 ||
      !std::isfinite(metric_volume) || metric_volume <= 0.0)
    return fail(ctx, BG_EINVAL, "Broyden geometry/shape");
  std::vector<double> w(n), scr(n);
  std::vector<int> sm(n);
  const double rs = std::cbrt(3.0 * volume / (4.0 * kPi * electrons));
  const double a = std::pow(12.0 / kPi, 2.0 / 3.0) / rs;
  for (int64_t i = 0; i < n; ++i) {
    const double g = g2[i];
    if (!std::isfinite(g) || g < 0.0) return fail(ctx, BG_EINVAL, "Broyden geometry/shape");
    sm[i] = smooth[i] ? 1 : 0;
    w[i] = (sm[i] && g > 0.0) ? 8.0 * kPi * metric_volume / g : 0.0;
    scr[i] = p.thomas_fermi ? g / (g + a) : 1.0;
  }
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
  auto m = std::make_unique<bg_mixer>();
  m->ctx = ctx;
  m->n = n;
  m->beta = p.beta;
  m->history = p.history;
  const size_t hn = (size_t)p.history * n;
  int rc;
  if ((rc = dalloc(m.get(), &m->prev_x, n)) || (rc = dalloc(m.get(), &m->prev_f, n)) ||
      (rc = dalloc(m.get(), &m->dx, hn)) || (rc = dalloc(m.get(), &m->df, hn)) ||
      (rc = dalloc(m.get(), &m->reduced, n)) || (rc = dalloc(m.get(), &m->w, n)) ||
      (rc = dalloc(m.get(), &m->screening, n)) || (rc = dalloc(m.get(), &m->smooth, n)) ||
      (rc = dalloc(m.get(), &m->forms, kMaxForms)) || (rc = dalloc(m.get(), &m->gamma, kMaxHistory)) ||
      (rc = dalloc(m.get(), &m->out, 8)) || (rc = dalloc(m.get(), &m->err, 4)))
    return rc;
  if ((e = cudaMemcpy(m->w, w.data(), sizeof(double) * n, cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(m->screening, scr.data(), sizeof(double) * n, cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(m->smooth, sm.data(), sizeof(int) * n, cudaMemcpyHostToDevice)) != cudaSuccess)
    return cuda_fail(ctx, e, "upload");
  if ((e = cudaMallocHost(&m->host_out, sizeof(double) * 40)) != cudaSuccess) return cuda_fail(ctx, e, "cudaMallocHost");
  if ((e = cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking)) != cudaSuccess)
    return cuda_fail(ctx, e, "cudaStreamCreate");
  m->own_stream = true;
  if ((e = cudaDeviceSynchronize()) != cudaSuccess) return cuda_fail(ctx, e, "mixer setup");
  *out = m.release();
  return BG_OK;
}

int bg_mixer_destroy(bg_mixer* m) {
  if (!m) return BG_OK;
  if (m->stream) cudaStreamSynchronize(m->stream);
  if (m->own_stream && m->stream) cudaStreamDestroy(m->stream);
  if (m->host_out) cudaFreeHost(m->host_out);
  delete m;
  return BG_OK;
}

int bg_mixer_set_stream(bg_mixer* m, void* stream) {
  if (!m) return BG_EINVAL;
  if (m->own_stream && m->stream) {
    cudaStreamSynchronize(m->stream);
    cudaStreamDestroy(m->stream);
  }
  m->own_stream = false;
  m->stream = static_cast<cudaStream_t>(stream);
  return BG_OK;
}

int bg_mixer_update(bg_mixer* m, const double* x, const double* f, double* next, int32_t ptr_kind,
                    bg_mixer_diagnostics* diag) {
  if (!m) return fail(nullptr, BG_EINVAL, "null mixer");
  bg_ctx* ctx = m->ctx;
  if (!x || !f || !next) return fail(ctx, BG_EINVAL, "null argument");
  if (ptr_kind != BG_PTR_HOST && ptr_kind != BG_PTR_DEVICE) return fail(ctx, BG_EINVAL, "pointer kind");
  if (m->failed) return fail(ctx, BG_EINVAL, "this mixer stopped at an earlier error");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
  const int64_t n = m->n;
  const size_t bytes = sizeof(double2) * n;
  const double2* dxp = reinterpret_cast<const double2*>(x);
  const double2* dfp = reinterpret_cast<const double2*>(f);
  double2* dnext = reinterpret_cast<double2*>(next);
  int rc;
  if (ptr_kind == BG_PTR_HOST) {
    if (!m->sx && ((rc = dalloc(m, &m->sx, n)) || (rc = dalloc(m, &m->sf, n)) || (rc = dalloc(m, &m->snext, n))))
      return rc;
    if ((e = cudaMemcpyAsync(m->sx, x, bytes, cudaMemcpyHostToDevice, m->stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(m->sf, f, bytes, cudaMemcpyHostToDevice, m->stream)) != cudaSuccess)
      return cuda_fail(ctx, e, "copy in");
    dxp = m->sx;
    dfp = m->sf;
    dnext = m->snext;
  }
  // crates/dft-engine/src/refscf/broyden.rs:328-351: slot (k-2) mod m from k = 2 on
  const int it = m->iteration + 1;
  const int slot = it > 1 ? (it - 2) % m->history : -1;
  const int p = std::min(std::max(it - 1, 0), m->history);
  const unsigned gb = grid_for(n);
  k_mix_diff<<<gb, 256, 0, m->stream>>>(dxp, dfp, m->prev_x, m->prev_f, m->dx + (slot < 0 ? 0 : (int64_t)slot * n),
                                        m->df + (slot < 0 ? 0 : (int64_t)slot * n), n, slot >= 0 ? 1 : 0);
  if (p > 0) {
    k_mix_forms<<<p * (p + 1) / 2 + p, kMixThreads, 0, m->stream>>>(m->df, n, p, dfp, m->w, m->forms);
    k_mix_solve<<<1, 32, 0, m->stream>>>(m->forms, p, m->gamma, m->out);
  }
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(ctx, e, "kernel launch");
  double* h = m->host_out;
  if (p > 0) {
    if ((e = cudaMemcpyAsync(h, m->out, sizeof(double) * 4, cudaMemcpyDeviceToHost, m->stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(m->stream)) != cudaSuccess)
      return cuda_fail(ctx, e, "mixer solve");
    if (h[0] != 0.0) {
      m->failed = true;
      m->iteration = it;
      char msg[160];
      if (h[0] == 2.0)
        std::snprintf(msg, sizeof msg, "nonfinite metric");
      else
        std::snprintf(msg, sizeof msg, "singular Broyden history at iteration %d: lambda_min %.6e, lambda_max %.6e", it,
                      h[1], h[2]);
      return fail(ctx, BG_EINVAL, msg);
    }
  }
  k_mix_apply<<<gb, 256, 0, m->stream>>>(dxp, dfp, m->dx, m->df, n, p, m->gamma, m->smooth, m->screening, m->beta,
                                         dnext, m->reduced, m->err);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(ctx, e, "kernel launch");
  if (ptr_kind == BG_PTR_HOST && (e = cudaMemcpyAsync(next, dnext, bytes, cudaMemcpyDeviceToHost, m->stream)) != cudaSuccess)
    return cuda_fail(ctx, e, "copy out");
  int* herr = reinterpret_cast<int*>(h + 4);
  if ((e = cudaMemcpyAsync(herr, m->err, sizeof(int), cudaMemcpyDeviceToHost, m->stream)) != cudaSuccess ||
      (e = cudaMemcpyAsync(h + 8, m->gamma, sizeof(double) * kMaxHistory, cudaMemcpyDeviceToHost, m->stream)) !=
          cudaSuccess ||
      (e = cudaStreamSynchronize(m->stream)) != cudaSuccess)
    return cuda_fail(ctx, e, "mixer update");
  m->iteration = it;
  m->occupancy = p;
  if (*herr) {
    cudaMemsetAsync(m->err, 0, sizeof(int), m->stream);
    cudaStreamSynchronize(m->stream);
    m->failed = true;
    return fail(ctx, BG_ENONFINITE, "nonfinite Broyden update");
  }
  if (diag) {
    double l2 = 0.0, mx = 0.0;
    for (int i = 0; i < p; ++i) {
      l2 += h[8 + i] * h[8 + i];
      mx = std::max(mx, std::fabs(h[8 + i]));
    }
    diag->iteration = it;
    diag->occupancy = p;
    diag->inserted_slot = slot;
    diag->gamma_l2 = std::sqrt(l2);
    diag->gamma_max = mx;
    diag->condition = p > 0 ? h[3] : 0.0;
  }
  return BG_OK;
}

int bg_mixer_gamma(const bg_mixer* m, double* gamma, int32_t* count) {
  if (!m || !gamma || !count) return BG_EINVAL;
  *count = m->occupancy;
  for (int i = 0; i < m->occupancy; ++i) gamma[i] = m->host_out[8 + i];
  return BG_OK;
}

int bg_mixer_reduced_residual(bg_mixer* m, double* out, int32_t ptr_kind) {
  if (!m || !out) return fail(m ? m->ctx : nullptr, BG_EINVAL, "null argument");
  const cudaMemcpyKind kind = ptr_kind == BG_PTR_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  cudaError_t e = cudaMemcpyAsync(out, m->reduced, sizeof(double2) * m->n, kind, m->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
  return e == cudaSuccess ? BG_OK : cuda_fail(m->ctx, e, "reduced residual");
}

int bg_mixer_metric(bg_mixer* m, const double* a, const double* b, double* out, int32_t ptr_kind) {
  if (!m || !a || !b || !out) return fail(m ? m->ctx : nullptr, BG_EINVAL, "null argument");
  bg_ctx* ctx = m->ctx;
  const int64_t n = m->n;
  const size_t bytes = sizeof(double2) * n;
  const double2* da = reinterpret_cast<const double2*>(a);
  const double2* db = reinterpret_cast<const double2*>(b);
  cudaError_t e = cudaSuccess;
  int rc;
  if (ptr_kind == BG_PTR_HOST) {
    if (!m->sx && ((rc = dalloc(m, &m->sx, n)) || (rc = dalloc(m, &m->sf, n)) || (rc = dalloc(m, &m->snext, n))))
      return rc;
    if ((e = cudaMemcpyAsync(m->sx, a, bytes, cudaMemcpyHostToDevice, m->stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(m->sf, b, bytes, cudaMemcpyHostToDevice, m->stream)) != cudaSuccess)
      return cuda_fail(ctx, e, "copy in");
    da = m->sx;
    db = m->sf;
  }
  // one form: <a, b> = the right-hand side slot of a p = 1 batch with dF_0 := a
  double* tmp = m->out + 4;
  k_mix_forms<<<1, kMixThreads, 0, m->stream>>>(da, n, 0, db, m->w, tmp);
  if ((e = cudaMemcpyAsync(m->host_out + 36, tmp, sizeof(double), cudaMemcpyDeviceToHost, m->stream)) != cudaSuccess ||
      (e = cudaStreamSynchronize(m->stream)) != cudaSuccess)
    return cuda_fail(ctx, e, "metric");
  *out = m->host_out[36];
  if (!std::isfinite(*out)) return fail(ctx, BG_ENONFINITE, "nonfinite metric");
  return BG_OK;
}

}  // extern "C"
