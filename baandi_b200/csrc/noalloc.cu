// bg_local_apply_noalloc: the local and kinetic part of H x for one k point, with every
// intermediate in a fixed scratch array that the library holds in device memory once its
// module is loaded on a device (with CUDA's default lazy module loading that happens at
// the first call on that device), so the call itself allocates nothing.
//
// Who needs it: callers whose device memory belongs to another runtime's pool (a
// framework caching allocator, an inference server's arena) or that run after an
// initialisation phase in which allocation is forbidden, because cudaMalloc/cudaFree
// may synchronise the device and stall unrelated streams.  They pass their own input
// and output buffers; the box of FFT values lives in g_noalloc_box below.
//
// Arithmetic: y = gather(FFT_fwd(V(r) . FFT_inv(scatter x))) / N + T x, the same
// operator as the local part of bg_op_apply_block, computed on the full n0 x n1 x n2
// box (no stick pruning) by line transforms along z, y and x in shared memory.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>

#include "bg_internal.h"
#include "fft_dev.cuh"

namespace bg {
namespace {

// 32 MiB of complex FP64: cols * n0 * n1 * n2 must not exceed kNoAllocBoxElems.
constexpr size_t kNoAllocBoxElems = (size_t)32 * 1024 * 1024 / sizeof(double2);
static __device__ __align__(256) double2 g_noalloc_box[kNoAllocBoxElems];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double2* g_box_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device (first call per device
// resolves it with cudaGetSymbolAddress; the host-side name is not a device address).
int scratch_for_current_device(double2** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    set_global_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    return BG_EDEVICE;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_box_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_box);
    if (e != cudaSuccess || !p) {
      set_global_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      return BG_EDEVICE;
    }
    g_box_ptr[dev] = static_cast<double2*>(p);
  }
  *out = g_box_ptr[dev];
  return BG_OK;
}

bool plan_for(int n, FftPlan* p) {
  if (n < 1 || n > 128) return false;
  p->n = n;
  p->nst = 0;
  int m = n;
  for (int r : {4, 2, 3, 5}) {
    while (m % r == 0) {
      if (p->nst == kMaxStages) return false;
      p->radix[p->nst++] = r;
      m /= r;
    }
  }
  if (m != 1) return false;
  for (int s = 0; s < p->nst; ++s)
    if (n / p->radix[s] > 32 * kButterfliesPerLane) return false;
  return true;
}

// Error bits of the last call, cleared by k_na_zero and read back by the host after the
// stream has finished: an fft_index entry outside [0, n0 n1 n2) (the access is skipped),
// a non-finite input coefficient.
constexpr int kErrIndex = 1, kErrNonfinite = 2;
static __device__ int g_noalloc_err;

__global__ void k_na_zero(double2* box, size_t n) {
  if (blockIdx.x == 0 && threadIdx.x == 0) g_noalloc_err = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    box[i] = make_double2(0.0, 0.0);
}

__global__ void k_na_scatter(double2* box, size_t nbox, const int32_t* __restrict__ idx, int64_t npw,
                             const double2* __restrict__ x, int64_t cols) {
  const size_t total = (size_t)npw * cols;
  int err = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t c = i / npw, g = i - c * npw;
    const int32_t f = idx[g];
    const double2 v = x[i];
    if (!isfinite(v.x) || !isfinite(v.y)) err |= kErrNonfinite;
    if (f < 0 || (size_t)f >= nbox) {
      err |= kErrIndex;
      continue;
    }
    box[c * nbox + f] = v;
  }
  if (err) atomicOr(&g_noalloc_err, err);
}

__global__ void k_na_multiply(double2* box, size_t nbox, const double* __restrict__ v, int64_t cols) {
  const size_t total = nbox * cols;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const double w = v[i % nbox];
    box[i].x *= w;
    box[i].y *= w;
  }
}

__global__ void k_na_gather(const double2* box, size_t nbox, const int32_t* __restrict__ idx, int64_t npw,
                            const double* __restrict__ kin, const double2* __restrict__ x, double2* y, int64_t cols,
                            double inv_n) {
  const size_t total = (size_t)npw * cols;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t c = i / npw, g = i - c * npw;
    const int32_t f = idx[g];
    // a row whose index is out of range has no grid value (flagged by the scatter pass)
    const double2 h = (f >= 0 && (size_t)f < nbox) ? box[c * nbox + f] : make_double2(0.0, 0.0);
    const double2 xv = x[i];
    y[i] = make_double2(h.x * inv_n + kin[g] * xv.x, h.y * inv_n + kin[g] * xv.y);
  }
}

struct Contig {
  int n;
  __device__ __forceinline__ int operator()(int l) const { return l * n; }
};

// Transform every line of one axis of the cols boxes: a block copies kLines lines to
// shared memory, runs the generic line FFT and writes them back.
constexpr int kLines = 16;
template <int SIGN>
__global__ void __launch_bounds__(256) k_na_lines(double2* box, size_t nbox, int64_t cols, int n, int64_t lines_per_box,
                                                  int64_t stride, int inner, int64_t inner_stride, FftPlan plan) {
  extern __shared__ double2 sm[];
  double2* tw = sm;
  double2* buf = sm + n;
  for (int q = threadIdx.x; q < n; q += blockDim.x) {
    double s, c;
    sincospi(2.0 * (double)q / (double)n, &s, &c);
    tw[q] = make_double2(c, s);
  }
  const int64_t total = lines_per_box * cols;
  const int64_t l0 = (int64_t)blockIdx.x * kLines;
  const int cnt = (int)(total - l0 < kLines ? total - l0 : kLines);
  if (cnt <= 0) return;
  // line l of box c starts at (l / inner) * inner_stride + (l % inner); elements `stride` apart
  auto start = [&](int64_t gl) -> size_t {
    const int64_t c = gl / lines_per_box, l = gl - c * lines_per_box;
    return (size_t)c * nbox + (size_t)((l / inner) * inner_stride + (l % inner));
  };
  for (int i = threadIdx.x; i < cnt * n; i += blockDim.x) {
    const int li = i / n, e = i - li * n;
    buf[li * n + e] = box[start(l0 + li) + (size_t)e * stride];
  }
  fft_lines<SIGN>(buf, cnt, Contig{n}, 1, plan, tw);
  for (int i = threadIdx.x; i < cnt * n; i += blockDim.x) {
    const int li = i / n, e = i - li * n;
    box[start(l0 + li) + (size_t)e * stride] = buf[li * n + e];
  }
}

template <int SIGN>
void lines_all_axes(double2* box, size_t nbox, int64_t cols, const int d[3], const FftPlan p[3], cudaStream_t s,
                    bool reverse) {
  for (int step = 0; step < 3; ++step) {
    const int axis = reverse ? step : 2 - step;
    const int n = d[axis];
    int64_t lines, stride, inner_stride;
    int inner;
    if (axis == 2) {  // z lines: contiguous
      lines = (int64_t)d[0] * d[1];
      stride = 1;
      inner = 1;
      inner_stride = d[2];
    } else if (axis == 1) {  // y lines at (x, z)
      lines = (int64_t)d[0] * d[2];
      stride = d[2];
      inner = d[2];
      inner_stride = (int64_t)d[1] * d[2];
    } else {  // x lines at (y, z)
      lines = (int64_t)d[1] * d[2];
      stride = (int64_t)d[1] * d[2];
      inner = d[1] * d[2];
      inner_stride = 0;
    }
    const int64_t blocks = (lines * cols + kLines - 1) / kLines;
    const size_t smem = sizeof(double2) * ((size_t)n + (size_t)kLines * n);
    k_na_lines<SIGN><<<(unsigned)blocks, 256, smem, s>>>(box, nbox, cols, n, lines, stride, inner, inner_stride,
                                                         p[axis]);
  }
}

}  // namespace
}  // namespace bg

using namespace bg;

extern "C" int bg_local_apply_noalloc(const int32_t dims[3], int64_t npw, const int32_t* fft_index,
                                      const double* v_grid, const double* kinetic, const double* x, double* y,
                                      int64_t cols, void* stream) {
  if (!dims || !fft_index || !v_grid || !kinetic || !x || !y) {
    set_global_error("null argument");
    return BG_EINVAL;
  }
  if (x == y) {
    set_global_error("x and y must be distinct buffers");
    return BG_EINVAL;
  }
  int d[3];
  FftPlan p[3];
  for (int i = 0; i < 3; ++i) {
    d[i] = dims[i];
    if (!plan_for(d[i], &p[i])) {
      set_global_error("grid lengths must be 2,3,5-smooth and at most 128");
      return BG_ESHAPE;
    }
  }
  const size_t nbox = (size_t)d[0] * d[1] * d[2];
  if (npw < 1 || cols < 0 || (size_t)npw > nbox) {
    set_global_error("row or column count out of range");
    return BG_ESHAPE;
  }
  if (cols > (int64_t)(kNoAllocBoxElems / nbox)) {
    set_global_error("cols * n0 * n1 * n2 exceeds the 32 MiB scratch of bg_local_apply_noalloc (2097152 complex values)");
    return BG_ESHAPE;
  }
  if (cols == 0) return BG_OK;
  double2* box = nullptr;
  int rc = scratch_for_current_device(&box);
  if (rc != BG_OK) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t nall = nbox * cols;
  const unsigned grid = (unsigned)std::min<size_t>((nall + 255) / 256, 148 * 16);
  k_na_zero<<<grid, 256, 0, s>>>(box, nall);
  k_na_scatter<<<grid, 256, 0, s>>>(box, nbox, fft_index, npw, reinterpret_cast<const double2*>(x), cols);
  lines_all_axes<1>(box, nbox, cols, d, p, s, false);
  k_na_multiply<<<grid, 256, 0, s>>>(box, nbox, v_grid, cols);
  lines_all_axes<-1>(box, nbox, cols, d, p, s, true);
  k_na_gather<<<grid, 256, 0, s>>>(box, nbox, fft_index, npw, kinetic, reinterpret_cast<const double2*>(x),
                                   reinterpret_cast<double2*>(y), cols, 1.0 / (double)nbox);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_global_error(std::string("kernel launch: ") + cudaGetErrorString(e));
    return BG_EDEVICE;
  }
  // The error word is read once the stream's work is done (a pageable copy: no allocation).
  int err = 0;
  e = cudaMemcpyFromSymbolAsync(&err, g_noalloc_err, sizeof(int), 0, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    set_global_error(std::string("bg_local_apply_noalloc: ") + cudaGetErrorString(e));
    return BG_EDEVICE;
  }
  if (err & kErrIndex) {
    set_global_error("fft_index holds an entry outside [0, n0*n1*n2); those rows were skipped");
    return BG_ESHAPE;
  }
  if (err & kErrNonfinite) {
    set_global_error("nonfinite input block");
    return BG_ENONFINITE;
  }
  return BG_OK;
}
