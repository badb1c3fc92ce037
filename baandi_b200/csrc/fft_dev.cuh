// Shared-memory line FFT engine for sm_100a (FP64 complex).
//
// A line of length n = r_0 r_1 ... r_{P-1} (radices 2, 3, 4, 5) is transformed by P
// in-place Stockham stages.  Stage s with radix R and span Ns (product of the earlier
// radices) reads element j + t n/R (t < R) of butterfly j, twiddles it by
// w^(t (j mod Ns) n/(Ns R)), does an R-point DFT and writes element
// (j / Ns) Ns R + (j mod Ns) + u Ns (u < R): the decimation-in-time autosort form, so
// no bit reversal is needed.  A warp owns whole lines within a stage: it loads every
// butterfly input of its lines into registers, __syncwarp, then writes the outputs
// into the same line, so the stage runs in place in shared memory.  Stages are
// separated by __syncthreads.
//
// Sign convention (docs/physics-conventions.md:61-78 of the reference): SIGN = +1 is
// the unscaled inverse f(r) = sum_G f(G) e^{+iGr}; SIGN = -1 the forward transform
// (scaling by 1/N is applied by the caller).
#pragma once
#include <cuda_runtime.h>

namespace bg {

constexpr int kMaxStages = 8;
constexpr int kButterfliesPerLane = 2;  // a line of n <= 128 fits one warp chunk at radix 2

struct FftPlan {
  int n;
  int nst;
  int radix[kMaxStages];
};

// Complex element types of the line transforms: double2 (FP64) and float2 (FP32).
template <class C>
struct Cplx;
template <>
struct Cplx<double2> {
  using R = double;
  __device__ __forceinline__ static double2 make(double x, double y) { return make_double2(x, y); }
};
template <>
struct Cplx<float2> {
  using R = float;
  __device__ __forceinline__ static float2 make(float x, float y) { return make_float2(x, y); }
};
template <class C>
using RealOf = typename Cplx<C>::R;
template <class C>
__device__ __forceinline__ C mkc(RealOf<C> x, RealOf<C> y) {
  return Cplx<C>::make(x, y);
}

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
template <int SIGN>
__device__ __forceinline__ float2 irot(float2 a) {
  return SIGN > 0 ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
// i * SIGN * a
template <int SIGN>
__device__ __forceinline__ double2 irot(double2 a) {
  return SIGN > 0 ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
}

template <int R, int SIGN>
__device__ __forceinline__ void dft(double2 (&v)[R]);

template <>
__device__ __forceinline__ void dft<2, 1>(double2 (&v)[2]) {
  const double2 a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}
template <>
__device__ __forceinline__ void dft<2, -1>(double2 (&v)[2]) {
  dft<2, 1>(v);
}

template <int SIGN>
__device__ __forceinline__ void dft3(double2 (&v)[3]) {
  const double h = 0.8660254037844386;  // sqrt(3)/2
  const double2 t1 = cadd(v[1], v[2]);
  const double2 t2 = make_double2(v[0].x - 0.5 * t1.x, v[0].y - 0.5 * t1.y);
  const double2 t3 = irot<SIGN>(cscale(csub(v[1], v[2]), h));
  v[0] = cadd(v[0], t1);
  v[1] = cadd(t2, t3);
  v[2] = csub(t2, t3);
}
template <>
__device__ __forceinline__ void dft<3, 1>(double2 (&v)[3]) { dft3<1>(v); }
template <>
__device__ __forceinline__ void dft<3, -1>(double2 (&v)[3]) { dft3<-1>(v); }

template <int SIGN>
__device__ __forceinline__ void dft4(double2 (&v)[4]) {
  const double2 a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
  const double2 c = cadd(v[1], v[3]), d = irot<SIGN>(csub(v[1], v[3]));
  v[0] = cadd(a, c);
  v[2] = csub(a, c);
  v[1] = cadd(b, d);
  v[3] = csub(b, d);
}
template <>
__device__ __forceinline__ void dft<4, 1>(double2 (&v)[4]) { dft4<1>(v); }
template <>
__device__ __forceinline__ void dft<4, -1>(double2 (&v)[4]) { dft4<-1>(v); }

template <int SIGN>
__device__ __forceinline__ void dft5(double2 (&v)[5]) {
  const double c1 = 0.30901699437494745, c2 = -0.8090169943749475;  // cos(2pi/5), cos(4pi/5)
  const double s1 = 0.9510565162951535, s2 = 0.5877852522924731;    // sin(2pi/5), sin(4pi/5)
  const double2 p1 = cadd(v[1], v[4]), m1 = csub(v[1], v[4]);
  const double2 p2 = cadd(v[2], v[3]), m2 = csub(v[2], v[3]);
  const double2 a1 = make_double2(v[0].x + c1 * p1.x + c2 * p2.x, v[0].y + c1 * p1.y + c2 * p2.y);
  const double2 a2 = make_double2(v[0].x + c2 * p1.x + c1 * p2.x, v[0].y + c2 * p1.y + c1 * p2.y);
  const double2 b1 = irot<SIGN>(make_double2(s1 * m1.x + s2 * m2.x, s1 * m1.y + s2 * m2.y));
  const double2 b2 = irot<SIGN>(make_double2(s2 * m1.x - s1 * m2.x, s2 * m1.y - s1 * m2.y));
  v[0] = cadd(v[0], cadd(p1, p2));
  v[1] = cadd(a1, b1);
  v[4] = csub(a1, b1);
  v[2] = cadd(a2, b2);
  v[3] = csub(a2, b2);
}
template <>
__device__ __forceinline__ void dft<5, 1>(double2 (&v)[5]) { dft5<1>(v); }
template <>
__device__ __forceinline__ void dft<5, -1>(double2 (&v)[5]) { dft5<-1>(v); }

// One stage over `nlines` lines.  Line `l` starts at base + off(l); consecutive line
// elements are `es` apart.  tw[q] = exp(+2 pi i q / n) (conjugated for SIGN = -1).
template <int R, int SIGN, class Off>
__device__ __forceinline__ void fft_stage(double2* base, int nlines, Off off, int es, int n, int ns,
                                          const double2* __restrict__ tw) {
  const int span = n / R;
  const int lpc = max(1, (32 * kButterfliesPerLane) / span);
  const int nchunks = (nlines + lpc - 1) / lpc;
  const int lane = threadIdx.x & 31;
  const int nw = blockDim.x >> 5;
  const int step = n / (ns * R);
  for (int c = threadIdx.x >> 5; c < nchunks; c += nw) {
    double2 v[kButterfliesPerLane][R];
    int jj[kButterfliesPerLane];
    double2* lp[kButterfliesPerLane];
#pragma unroll
    for (int q = 0; q < kButterfliesPerLane; ++q) {
      const int slot = lane + 32 * q;
      const int li = slot / span;
      const int j = slot - li * span;
      const int line = c * lpc + li;
      const bool act = (li < lpc) && (line < nlines);
      jj[q] = act ? j : -1;
      lp[q] = act ? base + off(line) : nullptr;
      if (act) {
#pragma unroll
        for (int t = 0; t < R; ++t) v[q][t] = lp[q][(j + t * span) * es];
      }
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < kButterfliesPerLane; ++q) {
      if (jj[q] >= 0) {
        const int j = jj[q];
        const int k = j % ns;
        if (ns > 1) {
#pragma unroll
          for (int t = 1; t < R; ++t) {
            double2 w = tw[t * k * step];
            if (SIGN < 0) w.y = -w.y;
            v[q][t] = cmul(v[q][t], w);
          }
        }
        dft<R, SIGN>(v[q]);
        const int o = (j / ns) * ns * R + k;
#pragma unroll
        for (int u = 0; u < R; ++u) lp[q][(o + u * ns) * es] = v[q][u];
      }
    }
    __syncwarp();
  }
}

// Full transform of `nlines` lines; begins and ends with __syncthreads.
template <int SIGN, class Off>
__device__ __forceinline__ void fft_lines(double2* base, int nlines, Off off, int es, const FftPlan& p,
                                          const double2* __restrict__ tw) {
  int ns = 1;
  for (int s = 0; s < p.nst; ++s) {
    __syncthreads();
    const int r = p.radix[s];
    if (r == 4)
      fft_stage<4, SIGN>(base, nlines, off, es, p.n, ns, tw);
    else if (r == 2)
      fft_stage<2, SIGN>(base, nlines, off, es, p.n, ns, tw);
    else if (r == 3)
      fft_stage<3, SIGN>(base, nlines, off, es, p.n, ns, tw);
    else
      fft_stage<5, SIGN>(base, nlines, off, es, p.n, ns, tw);
    ns *= r;
  }
  __syncthreads();
}

}  // namespace bg
