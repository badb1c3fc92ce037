// Hartree and LDA-PZ exchange-correlation fields of a density on the FFT box (FP64),
// the field step of one SCF map.
//
// Reference: crates/dft-engine/src/refscf/map.rs:41-198 (density -> rho(G) on the
// full grid with the 1/N to_reciprocal normalization, times 4 pi / |G|^2 with G = 0
// zero and the canonical Miller index of every grid point, back to real space; LDA-PZ
// on |rho|; E_H = dV/2 sum rho V_H, E_xc = dV sum |rho| eps_xc, and dV sum rho v_xc);
// crates/dft-physics/src/xc.rs:39-77 (Slater exchange and PZ81 correlation, zero at or
// below 1e-10); crates/dft-engine/src/refscf/density.rs:17-26 (|G|^2 of a Miller index).
//
// Kernels (one stream, fixed grids so that every sum is reduced in the same order):
//   k_f_xc       v_xc and eps_xc per point, the density as complex FFT input, block
//                partial sums of |rho| eps_xc and rho v_xc
//   k_f_lines    one axis of the 3D FFT: 16 lines of the axis per block in shared
//                memory (lines adjacent in memory, so loads and stores coalesce)
//   k_f_poisson  rho(G) / N x 4 pi / |G|^2
//   k_f_collect  V_H = Re(inverse), V_Hxc = V_H + v_xc, block sums of rho V_H
//   k_f_energies the three energies from the block sums in block order
#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

#include "op_internal.h"

namespace bg {
namespace {

constexpr int kLines = 16;
constexpr int kFieldBlocks = 4 * 148;
constexpr int kFieldThreads = 256;
constexpr double kDensityThreshold = 1e-10;
constexpr double kPi = 3.14159265358979323846;

struct Box3 {
  int n[3];
  int64_t total;
};

// LDA-PZ at a non-negative density a (Ha): eps_xc and v_xc.
__device__ __forceinline__ void lda_pz(double a, double* eps, double* v) {
  if (a <= kDensityThreshold) {
    *eps = 0.0;
    *v = 0.0;
    return;
  }
  const double rs = cbrt(3.0 / (4.0 * kPi)) / cbrt(a);
  const double eps_x = -0.75 * cbrt(3.0 / kPi) * cbrt(a);
  double eps_c, der;
  if (rs >= 1.0) {
    const double sq = sqrt(rs);
    const double den = 1.0 + 1.0529 * sq + 0.3334 * rs;
    eps_c = -0.1423 / den;
    der = 0.1423 * (1.0529 / (2.0 * sq) + 0.3334) / (den * den);
  } else {
    const double lr = log(rs);
    eps_c = 0.0311 * lr - 0.048 + 0.0020 * rs * lr - 0.0116 * rs;
    der = 0.0311 / rs + 0.0020 * (lr + 1.0) - 0.0116;
  }
  *eps = eps_x + eps_c;
  *v = 4.0 * eps_x / 3.0 + (eps_c - rs * der / 3.0);
}

// Sum of `v` over the block into sm (kFieldThreads doubles); thread 0 gets the total.
__device__ __forceinline__ double block_sum(double v, double* sm) {
  sm[threadIdx.x] = v;
  __syncthreads();
  for (int s = kFieldThreads / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) sm[threadIdx.x] += sm[threadIdx.x + s];
    __syncthreads();
  }
  const double r = sm[0];
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(kFieldThreads) k_f_xc(const double* __restrict__ rho, int64_t total,
                                                        double* __restrict__ vxc, double2* __restrict__ work,
                                                        double* __restrict__ part, int* err) {
  __shared__ double sm[kFieldThreads];
  double s_ex = 0.0, s_vx = 0.0;
  bool bad = false;
  for (int64_t p = blockIdx.x * (int64_t)kFieldThreads + threadIdx.x; p < total;
       p += (int64_t)gridDim.x * kFieldThreads) {
    const double d = rho[p];
    bad |= !isfinite(d);
    const double a = fabs(d);
    double eps, v;
    lda_pz(a, &eps, &v);
    vxc[p] = v;
    work[p] = make_double2(d, 0.0);
    s_ex += a * eps;
    s_vx += d * v;
  }
  if (bad) atomicOr(err, 1);
  s_ex = block_sum(s_ex, sm);
  s_vx = block_sum(s_vx, sm);
  if (threadIdx.x == 0) {
    part[3 * blockIdx.x + 1] = s_ex;
    part[3 * blockIdx.x + 2] = s_vx;
  }
}

// First element of line L of `axis` and the stride between its elements.
__device__ __forceinline__ int64_t line_base(const Box3& b, int axis, int64_t L, int64_t* stride) {
  if (axis == 2) {
    *stride = 1;
    return L * b.n[2];
  }
  if (axis == 1) {
    *stride = b.n[2];
    const int64_t x = L / b.n[2], z = L - x * b.n[2];
    return x * b.n[1] * (int64_t)b.n[2] + z;
  }
  *stride = (int64_t)b.n[1] * b.n[2];
  return L;
}

struct LinePitch {
  int ld;
  __device__ __forceinline__ int operator()(int l) const { return l * ld; }
};

template <int SIGN>
__global__ void __launch_bounds__(kFieldThreads) k_f_lines(double2* __restrict__ data, Box3 b, int axis, FftPlan plan,
                                                           const double2* __restrict__ twg) {
  extern __shared__ double2 fsm[];
  const int n = b.n[axis];
  const int ld = n | 1;
  double2* tw = fsm;
  double2* ln = fsm + n;
  const int64_t nlines = b.total / n;
  const int64_t L0 = (int64_t)blockIdx.x * kLines;
  const int cnt = nlines - L0 < kLines ? (int)(nlines - L0) : kLines;
  if (cnt <= 0) return;
  for (int i = threadIdx.x; i < n; i += blockDim.x) tw[i] = twg[i];
  int64_t stride;
  if (axis == 2) {
    const int64_t base = line_base(b, 2, L0, &stride);
    for (int e = threadIdx.x; e < cnt * n; e += blockDim.x) {
      const int l = e / n, i = e - l * n;
      ln[l * ld + i] = data[base + e];
    }
  } else {
    for (int e = threadIdx.x; e < cnt * n; e += blockDim.x) {
      const int i = e / cnt, l = e - i * cnt;
      const int64_t base = line_base(b, axis, L0 + l, &stride);
      ln[l * ld + i] = data[base + i * stride];
    }
  }
  fft_lines<SIGN>(ln, cnt, LinePitch{ld}, 1, plan, tw);
  if (axis == 2) {
    const int64_t base = line_base(b, 2, L0, &stride);
    for (int e = threadIdx.x; e < cnt * n; e += blockDim.x) {
      const int l = e / n, i = e - l * n;
      data[base + e] = ln[l * ld + i];
    }
  } else {
    for (int e = threadIdx.x; e < cnt * n; e += blockDim.x) {
      const int i = e / cnt, l = e - i * cnt;
      const int64_t base = line_base(b, axis, L0 + l, &stride);
      data[base + i * stride] = ln[l * ld + i];
    }
  }
}

struct Recip {
  double b[3][3];  // b[i][j]: Cartesian component i of reciprocal vector j (Bohr^-1)
};

__global__ void __launch_bounds__(kFieldThreads) k_f_poisson(double2* __restrict__ work, Box3 bx, Recip rc,
                                                             double inv_n) {
  for (int64_t p = blockIdx.x * (int64_t)kFieldThreads + threadIdx.x; p < bx.total;
       p += (int64_t)gridDim.x * kFieldThreads) {
    if (p == 0) {
      work[0] = make_double2(0.0, 0.0);
      continue;
    }
    const int64_t yz = (int64_t)bx.n[1] * bx.n[2];
    const int ijk[3] = {(int)(p / yz), (int)(p / bx.n[2] % bx.n[1]), (int)(p % bx.n[2])};
    double m[3];
    for (int a = 0; a < 3; ++a) m[a] = ijk[a] <= (bx.n[a] - 1) / 2 ? ijk[a] : ijk[a] - bx.n[a];
    double g2 = 0.0;
    for (int i = 0; i < 3; ++i) {
      const double gi = rc.b[i][0] * m[0] + rc.b[i][1] * m[1] + rc.b[i][2] * m[2];
      g2 += gi * gi;
    }
    const double k = 4.0 * kPi / g2;
    const double2 z = work[p];
    work[p] = make_double2(z.x * inv_n * k, z.y * inv_n * k);
  }
}

__global__ void __launch_bounds__(kFieldThreads) k_f_collect(const double2* __restrict__ work,
                                                             const double* __restrict__ rho,
                                                             const double* __restrict__ vxc, int64_t total,
                                                             double* __restrict__ v_h, double* __restrict__ v_hxc,
                                                             double* __restrict__ part) {
  __shared__ double sm[kFieldThreads];
  double s_eh = 0.0;
  for (int64_t p = blockIdx.x * (int64_t)kFieldThreads + threadIdx.x; p < total;
       p += (int64_t)gridDim.x * kFieldThreads) {
    const double vh = work[p].x;
    if (v_h) v_h[p] = vh;
    v_hxc[p] = vh + vxc[p];
    s_eh += rho[p] * vh;
  }
  s_eh = block_sum(s_eh, sm);
  if (threadIdx.x == 0) part[3 * blockIdx.x] = s_eh;
}

__global__ void k_f_energies(const double* __restrict__ part, int blocks, double dv, double* __restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s[3] = {0.0, 0.0, 0.0};
  for (int i = 0; i < blocks; ++i)
    for (int c = 0; c < 3; ++c) s[c] += part[3 * i + c];
  out[0] = 0.5 * dv * s[0];
  out[1] = dv * s[1];
  out[2] = dv * s[2];
}

// Density sphere transforms of the mixer (crates/dft-engine/src/refscf/density.rs:
// 173-237): forward picks FFT(rho)/N on the half-sphere indices; inverse forms
// 2 Re(sum_half c_G e^{iGr}) - Re c_0 from the half-sphere coefficients alone.
__global__ void k_f_load_real(const double* __restrict__ rho, int64_t total, double2* __restrict__ work) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < total; p += (int64_t)gridDim.x * blockDim.x)
    work[p] = make_double2(rho[p], 0.0);
}
__global__ void k_f_zero(double2* __restrict__ work, int64_t total) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < total; p += (int64_t)gridDim.x * blockDim.x)
    work[p] = make_double2(0.0, 0.0);
}
__global__ void k_f_pick(const double2* __restrict__ work, const int64_t* __restrict__ idx, int64_t n, double inv_n,
                         double2* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double2 z = work[idx[i]];
    out[i] = make_double2(z.x * inv_n, z.y * inv_n);
  }
}
__global__ void k_f_place(const double2* __restrict__ c, const int64_t* __restrict__ idx, int64_t n,
                          double2* __restrict__ work, int* err) {
  bool bad = false;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double2 z = c[i];
    bad |= !(isfinite(z.x) && isfinite(z.y));
    work[idx[i]] = z;
  }
  if (bad) atomicOr(err, 1);
}
__global__ void k_f_half_real(const double2* __restrict__ work, const double2* __restrict__ c, int64_t i0,
                              int64_t total, double* __restrict__ rho) {
  const double g0 = i0 >= 0 ? c[i0].x : 0.0;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < total; p += (int64_t)gridDim.x * blockDim.x)
    rho[p] = 2.0 * work[p].x - g0;
}

}  // namespace
}  // namespace bg

using namespace bg;

struct bg_fields {
  bg_ctx* ctx = nullptr;
  Box3 box{};
  Recip rc{};
  double volume = 0.0;
  FftPlan plan[3]{};
  double2* tw[3] = {nullptr, nullptr, nullptr};
  double2* work = nullptr;   // complex grid
  double* vxc = nullptr;
  double* part = nullptr;    // 3 sums per block
  double* energies = nullptr;
  double* stage_in = nullptr;   // host-pointer calls: density, v_hxc, v_h on the device
  double* stage_out = nullptr;
  double* stage_vh = nullptr;
  int* err = nullptr;
  int* err_host = nullptr;
  double* energies_host = nullptr;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::vector<std::unique_ptr<DevBuf>> bufs;
  // density half-sphere of the mixer
  int64_t nsphere = 0;
  int64_t sphere_g0 = -1;   // position of G = 0 in the sphere list
  int64_t* sphere = nullptr;
  double2* stage_c = nullptr;
};

namespace {

int falloc(bg_fields* f, size_t bytes, void** out) {
  auto b = std::make_unique<DevBuf>();
  b->bytes = bytes < 16 ? 16 : bytes;
  cudaError_t e = cudaMalloc(&b->p, b->bytes);
  if (e != cudaSuccess) return fail(f->ctx, BG_ENOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  *out = b->p;
  f->bufs.push_back(std::move(b));
  return BG_OK;
}

size_t lines_smem(int n) { return sizeof(double2) * ((size_t)n + (size_t)kLines * (n | 1)); }

}  // namespace

extern "C" {

int bg_fields_create(bg_ctx* ctx, const double rows[9], const int32_t dims[3], bg_fields** out) {
  if (!ctx || !rows || !dims || !out) return fail(ctx, BG_EINVAL, "null argument");
  Cell cell;
  if (cell_init(rows, &cell) != BG_OK) return fail(ctx, BG_ESHAPE, "lattice rows are singular or not finite");
  auto f = std::make_unique<bg_fields>();
  f->ctx = ctx;
  f->volume = cell.volume;
  int64_t total = 1;
  for (int a = 0; a < 3; ++a) {
    if (!make_fft_plan(dims[a], &f->plan[a]))
      return fail(ctx, BG_ESHAPE, "field grid lengths must be 2,3,5-smooth and at most 128");
    f->box.n[a] = dims[a];
    total *= dims[a];
  }
  f->box.total = total;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) f->rc.b[i][j] = cell.recip[i][j];
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
  void* vp;
  int rc;
  for (int a = 0; a < 3; ++a) {
    const std::vector<double> t = twiddles(dims[a]);
    if ((rc = falloc(f.get(), t.size() * sizeof(double), &vp))) return rc;
    f->tw[a] = static_cast<double2*>(vp);
    if ((e = cudaMemcpy(vp, t.data(), t.size() * sizeof(double), cudaMemcpyHostToDevice)) != cudaSuccess)
      return cuda_fail(ctx, e, "cudaMemcpy");
  }
  if ((rc = falloc(f.get(), sizeof(double2) * total, &vp))) return rc;
  f->work = static_cast<double2*>(vp);
  if ((rc = falloc(f.get(), sizeof(double) * total, &vp))) return rc;
  f->vxc = static_cast<double*>(vp);
  if ((rc = falloc(f.get(), sizeof(double) * 3 * kFieldBlocks, &vp))) return rc;
  f->part = static_cast<double*>(vp);
  if ((rc = falloc(f.get(), sizeof(double) * 4, &vp))) return rc;
  f->energies = static_cast<double*>(vp);
  if ((rc = falloc(f.get(), sizeof(int) * 4, &vp))) return rc;
  f->err = static_cast<int*>(vp);
  if ((e = cudaMemset(f->err, 0, sizeof(int) * 4)) != cudaSuccess) return cuda_fail(ctx, e, "cudaMemset");
  if ((e = cudaMallocHost(&f->err_host, sizeof(int) * 4)) != cudaSuccess) return cuda_fail(ctx, e, "cudaMallocHost");
  if ((e = cudaMallocHost(&f->energies_host, sizeof(double) * 4)) != cudaSuccess)
    return cuda_fail(ctx, e, "cudaMallocHost");
  size_t smem = 0;
  for (int a = 0; a < 3; ++a) smem = std::max(smem, lines_smem(dims[a]));
  if ((e = cudaFuncSetAttribute((const void*)k_f_lines<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) !=
          cudaSuccess ||
      (e = cudaFuncSetAttribute((const void*)k_f_lines<-1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) !=
          cudaSuccess)
    return cuda_fail(ctx, e, "cudaFuncSetAttribute");
  if ((e = cudaStreamCreateWithFlags(&f->stream, cudaStreamNonBlocking)) != cudaSuccess)
    return cuda_fail(ctx, e, "cudaStreamCreate");
  f->own_stream = true;
  *out = f.release();
  return BG_OK;
}

int bg_fields_destroy(bg_fields* f) {
  if (!f) return BG_OK;
  if (f->stream) cudaStreamSynchronize(f->stream);
  if (f->own_stream && f->stream) cudaStreamDestroy(f->stream);
  if (f->err_host) cudaFreeHost(f->err_host);
  if (f->energies_host) cudaFreeHost(f->energies_host);
  delete f;
  return BG_OK;
}

int bg_fields_set_stream(bg_fields* f, void* stream) {
  if (!f) return BG_EINVAL;
  if (f->own_stream && f->stream) {
    cudaStreamSynchronize(f->stream);
    cudaStreamDestroy(f->stream);
  }
  f->own_stream = false;
  f->stream = static_cast<cudaStream_t>(stream);
  return BG_OK;
}

int bg_fields_volume(const bg_fields* f, double* volume) {
  if (!f || !volume) return BG_EINVAL;
  *volume = f->volume;
  return BG_OK;
}

int bg_fields_lda_hartree(bg_fields* f, const double* density, double* v_hxc, double* v_h, double energies[3],
                          int32_t ptr_kind) {
  if (!f) return fail(nullptr, BG_EINVAL, "null fields object");
  bg_ctx* ctx = f->ctx;
  if (!density || !v_hxc || !energies) return fail(ctx, BG_EINVAL, "null argument");
  if (ptr_kind != BG_PTR_HOST && ptr_kind != BG_PTR_DEVICE) return fail(ctx, BG_EINVAL, "pointer kind");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
  const int64_t total = f->box.total;
  const size_t bytes = sizeof(double) * total;
  const double* rho = density;
  double* out = v_hxc;
  double* vh = v_h;
  int rc;
  void* vp;
  if (ptr_kind == BG_PTR_HOST) {
    if (!f->stage_in) {
      if ((rc = falloc(f, bytes, &vp))) return rc;
      f->stage_in = static_cast<double*>(vp);
      if ((rc = falloc(f, bytes, &vp))) return rc;
      f->stage_out = static_cast<double*>(vp);
      if ((rc = falloc(f, bytes, &vp))) return rc;
      f->stage_vh = static_cast<double*>(vp);
    }
    if ((e = cudaMemcpyAsync(f->stage_in, density, bytes, cudaMemcpyHostToDevice, f->stream)) != cudaSuccess)
      return cuda_fail(ctx, e, "copy in");
    rho = f->stage_in;
    out = f->stage_out;
    vh = v_h ? f->stage_vh : nullptr;
  }
  const Box3 b = f->box;
  k_f_xc<<<kFieldBlocks, kFieldThreads, 0, f->stream>>>(rho, total, f->vxc, f->work, f->part, f->err);
  for (int a = 2; a >= 0; --a) {
    const int blocks = (int)((total / b.n[a] + kLines - 1) / kLines);
    k_f_lines<-1><<<blocks, kFieldThreads, lines_smem(b.n[a]), f->stream>>>(f->work, b, a, f->plan[a], f->tw[a]);
  }
  k_f_poisson<<<kFieldBlocks, kFieldThreads, 0, f->stream>>>(f->work, b, f->rc, 1.0 / (double)total);
  for (int a = 0; a < 3; ++a) {
    const int blocks = (int)((total / b.n[a] + kLines - 1) / kLines);
    k_f_lines<1><<<blocks, kFieldThreads, lines_smem(b.n[a]), f->stream>>>(f->work, b, a, f->plan[a], f->tw[a]);
  }
  k_f_collect<<<kFieldBlocks, kFieldThreads, 0, f->stream>>>(f->work, rho, f->vxc, total, vh, out, f->part);
  k_f_energies<<<1, 32, 0, f->stream>>>(f->part, kFieldBlocks, f->volume / (double)total, f->energies);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(ctx, e, "kernel launch");
  if ((e = cudaMemcpyAsync(f->energies_host, f->energies, sizeof(double) * 3, cudaMemcpyDeviceToHost, f->stream)) !=
          cudaSuccess ||
      (e = cudaMemcpyAsync(f->err_host, f->err, sizeof(int), cudaMemcpyDeviceToHost, f->stream)) != cudaSuccess)
    return cuda_fail(ctx, e, "copy out");
  if ((e = cudaStreamSynchronize(f->stream)) != cudaSuccess) return cuda_fail(ctx, e, "fields");
  if (f->err_host[0]) {
    cudaMemsetAsync(f->err, 0, sizeof(int), f->stream);
    cudaStreamSynchronize(f->stream);
    return fail(ctx, BG_ENONFINITE, "non-finite density value");
  }
  for (int i = 0; i < 3; ++i)
    if (!std::isfinite(f->energies_host[i])) return fail(ctx, BG_ENONFINITE, "field energy not representable");
  if (ptr_kind == BG_PTR_HOST) {
    if ((e = cudaMemcpyAsync(v_hxc, out, bytes, cudaMemcpyDeviceToHost, f->stream)) != cudaSuccess)
      return cuda_fail(ctx, e, "copy out");
    if (v_h && (e = cudaMemcpyAsync(v_h, vh, bytes, cudaMemcpyDeviceToHost, f->stream)) != cudaSuccess)
      return cuda_fail(ctx, e, "copy out");
    if ((e = cudaStreamSynchronize(f->stream)) != cudaSuccess) return cuda_fail(ctx, e, "copy out");
  }
  for (int i = 0; i < 3; ++i) energies[i] = f->energies_host[i];
  return BG_OK;
}

int bg_fields_set_sphere(bg_fields* f, int64_t n, const int64_t* flat_index) {
  if (!f || !flat_index || n < 1) return fail(f ? f->ctx : nullptr, BG_EINVAL, "argument");
  if (f->sphere) return fail(f->ctx, BG_EINVAL, "the density sphere is already set");
  int64_t g0 = -1;
  for (int64_t i = 0; i < n; ++i) {
    if (flat_index[i] < 0 || flat_index[i] >= f->box.total) return fail(f->ctx, BG_ESHAPE, "sphere index outside the box");
    if (flat_index[i] == 0) g0 = i;
  }
  cudaError_t e = cudaSetDevice(f->ctx->device);
  if (e != cudaSuccess) return cuda_fail(f->ctx, e, "cudaSetDevice");
  void* vp;
  int rc;
  if ((rc = falloc(f, sizeof(int64_t) * n, &vp))) return rc;
  f->sphere = static_cast<int64_t*>(vp);
  if ((rc = falloc(f, sizeof(double2) * n, &vp))) return rc;
  f->stage_c = static_cast<double2*>(vp);
  if ((e = cudaMemcpy(f->sphere, flat_index, sizeof(int64_t) * n, cudaMemcpyHostToDevice)) != cudaSuccess)
    return cuda_fail(f->ctx, e, "upload");
  f->nsphere = n;
  f->sphere_g0 = g0;
  return BG_OK;
}

static void f_transform(bg_fields* f, int sign) {
  const Box3 b = f->box;
  for (int i = 0; i < 3; ++i) {
    const int a = sign < 0 ? 2 - i : i;
    const int blocks = (int)((b.total / b.n[a] + kLines - 1) / kLines);
    if (sign < 0)
      k_f_lines<-1><<<blocks, kFieldThreads, lines_smem(b.n[a]), f->stream>>>(f->work, b, a, f->plan[a], f->tw[a]);
    else
      k_f_lines<1><<<blocks, kFieldThreads, lines_smem(b.n[a]), f->stream>>>(f->work, b, a, f->plan[a], f->tw[a]);
  }
}

int bg_fields_sphere_forward(bg_fields* f, const double* density, double* coeffs, int32_t ptr_kind) {
  if (!f || !density || !coeffs) return fail(f ? f->ctx : nullptr, BG_EINVAL, "null argument");
  bg_ctx* ctx = f->ctx;
  if (!f->sphere) return fail(ctx, BG_EINVAL, "set the density sphere first");
  if (ptr_kind != BG_PTR_HOST && ptr_kind != BG_PTR_DEVICE) return fail(ctx, BG_EINVAL, "pointer kind");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
  const int64_t total = f->box.total;
  const double* rho = density;
  double2* out = reinterpret_cast<double2*>(coeffs);
  void* vp;
  int rc;
  if (ptr_kind == BG_PTR_HOST) {
    if (!f->stage_in) {
      if ((rc = falloc(f, sizeof(double) * total, &vp))) return rc;
      f->stage_in = static_cast<double*>(vp);
      if ((rc = falloc(f, sizeof(double) * total, &vp))) return rc;
      f->stage_out = static_cast<double*>(vp);
      if ((rc = falloc(f, sizeof(double) * total, &vp))) return rc;
      f->stage_vh = static_cast<double*>(vp);
    }
    if ((e = cudaMemcpyAsync(f->stage_in, density, sizeof(double) * total, cudaMemcpyHostToDevice, f->stream)) !=
        cudaSuccess)
      return cuda_fail(ctx, e, "copy in");
    rho = f->stage_in;
    out = f->stage_c;
  }
  const unsigned g = (unsigned)std::min<int64_t>((total + 255) / 256, kFieldBlocks);
  k_f_load_real<<<g, 256, 0, f->stream>>>(rho, total, f->work);
  f_transform(f, -1);
  const unsigned gs = (unsigned)std::min<int64_t>((f->nsphere + 255) / 256, kFieldBlocks);
  k_f_pick<<<gs, 256, 0, f->stream>>>(f->work, f->sphere, f->nsphere, 1.0 / (double)total, out);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(ctx, e, "kernel launch");
  if (ptr_kind == BG_PTR_HOST &&
      (e = cudaMemcpyAsync(coeffs, out, sizeof(double2) * f->nsphere, cudaMemcpyDeviceToHost, f->stream)) != cudaSuccess)
    return cuda_fail(ctx, e, "copy out");
  if ((e = cudaStreamSynchronize(f->stream)) != cudaSuccess) return cuda_fail(ctx, e, "sphere forward");
  return BG_OK;
}

int bg_fields_sphere_inverse(bg_fields* f, const double* coeffs, double* density, int32_t ptr_kind) {
  if (!f || !density || !coeffs) return fail(f ? f->ctx : nullptr, BG_EINVAL, "null argument");
  bg_ctx* ctx = f->ctx;
  if (!f->sphere) return fail(ctx, BG_EINVAL, "set the density sphere first");
  if (ptr_kind != BG_PTR_HOST && ptr_kind != BG_PTR_DEVICE) return fail(ctx, BG_EINVAL, "pointer kind");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
  const int64_t total = f->box.total;
  const double2* c = reinterpret_cast<const double2*>(coeffs);
  double* rho = density;
  void* vp;
  int rc;
  if (ptr_kind == BG_PTR_HOST) {
    if (!f->stage_in) {
      if ((rc = falloc(f, sizeof(double) * total, &vp))) return rc;
      f->stage_in = static_cast<double*>(vp);
      if ((rc = falloc(f, sizeof(double) * total, &vp))) return rc;
      f->stage_out = static_cast<double*>(vp);
      if ((rc = falloc(f, sizeof(double) * total, &vp))) return rc;
      f->stage_vh = static_cast<double*>(vp);
    }
    if ((e = cudaMemcpyAsync(f->stage_c, coeffs, sizeof(double2) * f->nsphere, cudaMemcpyHostToDevice, f->stream)) !=
        cudaSuccess)
      return cuda_fail(ctx, e, "copy in");
    c = f->stage_c;
    rho = f->stage_out;
  }
  const unsigned g = (unsigned)std::min<int64_t>((total + 255) / 256, kFieldBlocks);
  const unsigned gs = (unsigned)std::min<int64_t>((f->nsphere + 255) / 256, kFieldBlocks);
  k_f_zero<<<g, 256, 0, f->stream>>>(f->work, total);
  k_f_place<<<gs, 256, 0, f->stream>>>(c, f->sphere, f->nsphere, f->work, f->err);
  f_transform(f, 1);
  k_f_half_real<<<g, 256, 0, f->stream>>>(f->work, c, f->sphere_g0, total, rho);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(ctx, e, "kernel launch");
  if (ptr_kind == BG_PTR_HOST &&
      (e = cudaMemcpyAsync(density, rho, sizeof(double) * total, cudaMemcpyDeviceToHost, f->stream)) != cudaSuccess)
    return cuda_fail(ctx, e, "copy out");
  if ((e = cudaMemcpyAsync(f->err_host, f->err, sizeof(int), cudaMemcpyDeviceToHost, f->stream)) != cudaSuccess ||
      (e = cudaStreamSynchronize(f->stream)) != cudaSuccess)
    return cuda_fail(ctx, e, "sphere inverse");
  if (f->err_host[0]) {
    cudaMemsetAsync(f->err, 0, sizeof(int), f->stream);
    cudaStreamSynchronize(f->stream);
    return fail(ctx, BG_ENONFINITE, "non-finite density coefficient");
  }
  return BG_OK;
}

}  // extern "C"
