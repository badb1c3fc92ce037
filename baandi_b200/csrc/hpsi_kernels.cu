// sm_100a kernels of the Hamiltonian apply H.x (FP64).
//
// Local part, three passes over a stick buffer in HBM (layout [unit][z][stick]):
//   k_sticks_inverse  scatter the sphere coefficients of one stick group into zeroed
//                     z lines in shared memory (Gamma: pack two ORC columns into one
//                     complex vector), inverse FFT along z, store [z][stick].
//   k_planes          one (unit, z) plane in shared memory: inverse FFT along y on
//                     the x rows holding sticks, along x on every column, times V(r),
//                     forward x, forward y, store the stick values back.
//   k_sticks_forward  forward FFT along z, x 1/N, gather to the sphere and add the
//                     kinetic term (Gamma: unpack the pair into two ORC columns).
// Nonlocal part, y += P (D (P^H x)):
//   k_project         split-K partial products of P^H X (P^T X on Gamma ORC rows)
//   k_couple          ordered sum of the partials and the per-atom D blocks
//   k_back            y += P W
//
// Reference (paths inside the reference project): crates/dft-solvers/src/
// distributed_fft.rs:837-1130, 1198-1288 (scatter, pruned transforms, x V, 1/N,
// gather); crates/dft-physics/src/distributed_complex.rs:340-386 (complex apply);
// crates/dft-physics/src/distributed_real_gamma.rs:654-689 (pair pack), :1307-1347
// (unpack + kinetic), :957-1017, 1184-1248 (nonlocal).
#include "hpsi.h"
#include "gemm_tc.cuh"
#include "fft_fast.cuh"
#include "gemm_tiles.cuh"

#include <algorithm>

namespace bg {

namespace {

constexpr double kSqrt2 = 1.4142135623730951;
constexpr double kInvSqrt2 = 0.7071067811865476;

struct LineOffStride {
  int stride;
  __device__ __forceinline__ int operator()(int l) const { return l * stride; }
};
struct LineOffRows {
  const int* rows;
  int pitch;
  __device__ __forceinline__ int operator()(int l) const { return rows[l] * pitch; }
};
// The fast plane kernel stages V(r) of its plane in shared memory when plane and
// potential fit together (N <= 90: 90 x 91 x 16 + 90 x 90 x 8 bytes = 196 KB).
__host__ __device__ constexpr bool v_in_smem(int n) { return n <= 90; }
// FP32 planes are half the size: V(r) fits beside them up to N = 128.
template <class C>
__host__ __device__ constexpr bool v_in_smem_t(int n) {
  return sizeof(C) == sizeof(double2) ? v_in_smem(n) : n <= 128;
}

struct LineOffTable {
  const int* off;
  __device__ __forceinline__ int operator()(int l) const { return off[l]; }
};
struct LineOffCols {
  __device__ __forceinline__ int operator()(int l) const { return l; }
};

__device__ __forceinline__ bool finite2(double a, double b) { return isfinite(a) && isfinite(b); }

// FP64 (double2) or FP32 (float2) local apply: twiddles, stick buffer and potential of
// the element type.  The FP32 stick buffer reuses the FP64 one's memory.
template <class C>
__device__ __forceinline__ const C* tw_axis(const BoxGeo& g, int axis);
template <>
__device__ __forceinline__ const double2* tw_axis<double2>(const BoxGeo& g, int axis) {
  return axis == 0 ? g.tw0 : axis == 1 ? g.tw1 : g.tw2;
}
template <>
__device__ __forceinline__ const float2* tw_axis<float2>(const BoxGeo& g, int axis) {
  return axis == 0 ? g.tw0f : axis == 1 ? g.tw1f : g.tw2f;
}
template <class C>
__device__ __forceinline__ C* sticks_of(const OpTables& t) {
  return reinterpret_cast<C*>(t.sbuf);
}
template <class C>
__device__ __forceinline__ C to_elem(double x, double y) {
  return mkc<C>(RealOf<C>(x), RealOf<C>(y));
}

// ---------------------------------------------------------------- pass 1
// Blocks of the stick kernels per SM from their shared memory (twiddles and 32 lines of
// pitch N|1), at most 8: more groups in flight keep more stick rows moving.
template <int N, class C>
constexpr int sticks_blocks_per_sm() {
  if (N == 0) return 1;
  const int bytes = (int)sizeof(C) * (N + 32 * (N | 1));
  const int fit = 233472 / (bytes + 1024);
  return fit < 1 ? 1 : (fit > 8 ? 8 : fit);
}

template <bool GAMMA, int N, class C = double2>
__global__ void __launch_bounds__(N == 0 ? 256 : 128, sticks_blocks_per_sm<N, C>()) k_sticks_inverse(const OpTables* __restrict__ tabs, BoxGeo g, Batch b) {
  static_assert(N != 0 || sizeof(C) == sizeof(double2), "the runtime-plan engine is FP64 only");
  const OpTables& t = tabs[blockIdx.z];
  const CallArgs a = resolve(b.a[blockIdx.z]);
  const int grp = blockIdx.x, unit = blockIdx.y;
  if (grp >= t.ngroups || unit >= a.units) return;
  extern __shared__ __align__(16) unsigned char si_raw[];
  C* tw = reinterpret_cast<C*>(si_raw);
  C* st = tw + g.n2;
  const int s0 = t.grp_stick[grp], cnt = t.grp_stick[grp + 1] - s0;
  const C* twg = tw_axis<C>(g, 2);
  for (int i = threadIdx.x; i < g.n2; i += blockDim.x) tw[i] = twg[i];
  for (int i = threadIdx.x; i < cnt * g.ld2; i += blockDim.x) st[i] = to_elem<C>(0.0, 0.0);
  __syncthreads();
  const int e0 = t.grp_entry[grp], e1 = t.grp_entry[grp + 1];
  bool bad = false;
  if (!GAMMA) {
    const double2* x = reinterpret_cast<const double2*>(a.x + (int64_t)unit * a.ldx);
    // unrolled so that several entry-then-value load chains are in flight per thread
#pragma unroll 4
    for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
      const int2 en = t.entries[e];
      const double2 v = x[en.x];
      bad |= !finite2(v.x, v.y);
      st[en.y] = to_elem<C>(v.x, v.y);
    }
  } else {
    const int ca = 2 * unit;
    const bool hasb = ca + 1 < a.cols;
    const double* xa = a.x + (int64_t)ca * a.ldx;
    const double* xb = a.x + (int64_t)(hasb ? ca + 1 : ca) * a.ldx;
#pragma unroll 4
    for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
      const int2 en = t.entries[e];
      const int code = en.x;
      double2 v;
      if (code == 0) {
        v = make_double2(xa[0], hasb ? xb[0] : 0.0);
      } else {
        const int r = code > 0 ? code : -code;
        const double2 pa = make_double2(xa[r] * kInvSqrt2, xa[r + 1] * kInvSqrt2);
        const double2 pb = hasb ? make_double2(xb[r] * kInvSqrt2, xb[r + 1] * kInvSqrt2) : make_double2(0.0, 0.0);
        // plus: a + i b ; minus: conj(a) + i conj(b)
        v = code > 0 ? make_double2(pa.x - pb.y, pa.y + pb.x) : make_double2(pa.x + pb.y, -pa.y + pb.x);
      }
      bad |= !finite2(v.x, v.y);
      st[en.y] = to_elem<C>(v.x, v.y);
    }
  }
  if (bad) atomicOr(t.err, 1);
  if constexpr (N == 0) {
    fft_lines<1>(st, cnt, LineOffStride{g.ld2}, 1, g.p2, tw);
  } else {
    __syncthreads();
    fast::pass<N, 1, 1>(st, cnt, LineOffStride{fast::pitch_of<N>()}, tw);
  }
  C* out = sticks_of<C>(t) + (int64_t)unit * g.n2 * t.S + s0;
  for (int i = threadIdx.x; i < cnt * g.n2; i += blockDim.x) {
    const int z = i / cnt, sl = i - z * cnt;
    out[(int64_t)z * t.S + sl] = st[sl * g.ld2 + z];
  }
}

// ---------------------------------------------------------------- pass 2
__global__ void __launch_bounds__(512) k_planes(const OpTables* __restrict__ tabs, BoxGeo g, Batch b) {
  const OpTables& t = tabs[blockIdx.z];
  const CallArgs a = resolve(b.a[blockIdx.z]);
  const int unit = blockIdx.x, z = blockIdx.y;
  if (unit >= a.units) return;
  extern __shared__ double2 sm[];
  double2* tw0 = sm;
  double2* tw1 = tw0 + g.n0;
  double2* pl = tw1 + g.n1;
  for (int i = threadIdx.x; i < g.n0; i += blockDim.x) tw0[i] = g.tw0[i];
  for (int i = threadIdx.x; i < g.n1; i += blockDim.x) tw1[i] = g.tw1[i];
  const int np = g.n0 * g.pitch;
  for (int i = threadIdx.x; i < np; i += blockDim.x) pl[i] = make_double2(0.0, 0.0);
  __syncthreads();
  double2* row = t.sbuf + ((int64_t)unit * g.n2 + z) * t.S;
  for (int s = threadIdx.x; s < t.S; s += blockDim.x) pl[t.stick_plane[s]] = row[s];
  // inverse: y on the occupied x rows, x on every column
  fft_lines<1>(pl, t.nxact, LineOffRows{t.xact, g.pitch}, 1, g.p1, tw1);
  fft_lines<1>(pl, g.n1, LineOffCols{}, g.pitch, g.p0, tw0);
  const double* v = (a.vt ? a.vt : t.vt) + (int64_t)z * g.vstride;
  for (int i = threadIdx.x; i < g.n0 * g.n1; i += blockDim.x) {
    const int y = i / g.n0, x = i - y * g.n0;
    const double w = v[i];
    double2& p = pl[x * g.pitch + y];
    p.x *= w;
    p.y *= w;
  }
  fft_lines<-1>(pl, g.n1, LineOffCols{}, g.pitch, g.p0, tw0);
  fft_lines<-1>(pl, t.nxact, LineOffRows{t.xact, g.pitch}, 1, g.p1, tw1);
  for (int s = threadIdx.x; s < t.S; s += blockDim.x) row[s] = pl[t.stick_plane[s]];
}

// Cubic grids with a compile-time two-stage plan (R1, R2).  One block per (unit, z
// plane, k):
//   y inverse  on the x rows that hold sticks: the first stage reads its butterflies'
//              inputs straight from the stick row in global memory (zero where the plane
//              has no stick), the second stage runs in the shared-memory plane
//   x pass     on every column y: inverse, x V(r), forward with the middle in registers;
//              inputs outside the stick rows are zero and not loaded, outputs are kept
//              only in the stick rows
//   y forward  on the stick rows: the last stage writes the stick positions straight
//              back to the stick row
// The plane is never cleared or scattered: every element a pass reads was written by
// the pass before it in the same block.
// Blocks of k_planes_fast that fit an SM's 228 KB of shared memory (1 KB reserved per
// block), at most 4: the register budget per thread follows from it.
template <int N, class C>
__host__ __device__ constexpr int planes_blocks_per_sm() {
  const int P = N | 1;
  const int bytes = (int)sizeof(C) * (N + N * P) + (v_in_smem_t<C>(N) ? (int)sizeof(C) / 2 * N * N : 0) + 4 * N;
  const int fit = 233472 / (bytes + 1024);
  return fit < 1 ? 1 : (fit > 4 ? 4 : fit);
}
// Threads of a k_planes_fast block: 16 warps where the plane allows one block per SM
// (108^3: the block alone must hide the latencies), else 8.
template <int N, class C>
__host__ __device__ constexpr int planes_threads() {
  return planes_blocks_per_sm<N, C>() == 1 ? 512 : 256;
}

template <int N, class C = double2>
__global__ void __launch_bounds__(planes_threads<N, C>(), planes_blocks_per_sm<N, C>())
    k_planes_fast(const OpTables* __restrict__ tabs, BoxGeo g, Batch b) {
  using T = RealOf<C>;
  using Pl = fast::Plan<N>;
  static_assert(Pl::nst == 2, "two-stage plans");
  constexpr int R1 = Pl::radix[0], R2 = Pl::radix[1];
  const OpTables& t = tabs[blockIdx.z];
  const CallArgs a = resolve(b.a[blockIdx.z]);
  const int unit = blockIdx.x, z = blockIdx.y;
  if (unit >= a.units) return;
  constexpr int P = fast::pitch_of<N>();
  constexpr bool VS = v_in_smem_t<C>(N);
  constexpr int EPC = 16 / (int)sizeof(T);  // potential values per 16-byte copy
  extern __shared__ __align__(16) unsigned char pf_raw[];
  C* tw = reinterpret_cast<C*>(pf_raw);
  C* pl = tw + N;
  T* vs = reinterpret_cast<T*>(pl + N * P);   // V(r) of this plane, [y][x]
  int* rows = reinterpret_cast<int*>(vs + (VS ? N * N : 0));
  const int nx = t.nxact;
  // V(r) of the plane arrives asynchronously while the y pass runs (16-byte cp.async;
  // the plane strides keep every plane 16-byte aligned)
  const T* v;
  if constexpr (sizeof(T) == sizeof(double))
    v = reinterpret_cast<const T*>((a.vt ? a.vt : t.vt) + (int64_t)z * g.vstride);
  else
    v = reinterpret_cast<const T*>(t.vtf + (int64_t)z * g.vstridef);
  if constexpr (VS) {
    const unsigned dst = static_cast<unsigned>(__cvta_generic_to_shared(vs));
    for (int i = threadIdx.x; i < N * N / EPC; i += blockDim.x)
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst + 16u * i), "l"(v + EPC * i));
    for (int i = (N * N / EPC) * EPC + threadIdx.x; i < N * N; i += blockDim.x) vs[i] = v[i];
    asm volatile("cp.async.commit_group;\n" ::);
  }
  const C* twg = tw_axis<C>(g, 0);
  for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = twg[i];
  for (int i = threadIdx.x; i < nx; i += blockDim.x) rows[i] = t.xact[i] * P;
  __syncthreads();
  fast::StageIo<C> io;
  io.tab = t.line_stick;
  io.row = sticks_of<C>(t) + ((int64_t)unit * N + z) * t.S;
  io.xb = t.xbits;
  const int lane = threadIdx.x & 31;
  int first, count;
  constexpr int kWarps = planes_threads<N, C>() / 32;
  // stick rows per warp (read again for the last pass rather than kept live across the x pass)
  fast::owned_block(nx, kWarps == 16 ? t.yper16 : t.yper, &first, &count);
  if (count > 0) {
    fast::stage<N, R1, 1, 1, 1, fast::kInGlobal>(pl, first, count, LineOffTable{rows}, tw, lane, io);
    fast::stage<N, R2, R1, 1, 1>(pl, first, count, LineOffTable{rows}, tw, lane);
  }
  asm volatile("cp.async.wait_all;\n" ::);
  __syncthreads();
  {
    int xf, xc;
    constexpr int xper = fast::balanced_lines<N, 2, 1>(N, kWarps);
    fast::owned_block(N, xper, &xf, &xc);
    if (xc > 0) {
      // line = column y, element = x: weight V(x, y, z)
      auto wgt = [&](int y, int x) -> T { return VS ? vs[y * N + x] : v[y * N + x]; };
      fast::inverse_weight_forward<N, P, true>(pl, xf, xc, LineOffCols{}, tw, wgt, lane, io);
    }
  }
  __syncthreads();
  fast::owned_block(nx, kWarps == 16 ? t.yper16 : t.yper, &first, &count);
  if (count > 0) {
    fast::stage<N, R1, 1, -1, 1>(pl, first, count, LineOffTable{rows}, tw, lane);
    fast::stage<N, R2, R1, -1, 1, fast::kOutGlobal>(pl, first, count, LineOffTable{rows}, tw, lane, io);
  }
}

// ---------------------------------------------------------------- pass 3
template <bool GAMMA, int N, class C = double2>
__global__ void __launch_bounds__(N == 0 ? 256 : 128, sticks_blocks_per_sm<N, C>()) k_sticks_forward(const OpTables* __restrict__ tabs, BoxGeo g, Batch b) {
  static_assert(N != 0 || sizeof(C) == sizeof(double2), "the runtime-plan engine is FP64 only");
  const OpTables& t = tabs[blockIdx.z];
  const CallArgs a = resolve(b.a[blockIdx.z]);
  const int grp = blockIdx.x, unit = blockIdx.y;
  if (grp >= t.ngroups || unit >= a.units) return;
  extern __shared__ __align__(16) unsigned char sf_raw[];
  C* tw = reinterpret_cast<C*>(sf_raw);
  C* st = tw + g.n2;
  const int s0 = t.grp_stick[grp], cnt = t.grp_stick[grp + 1] - s0;
  const C* twg = tw_axis<C>(g, 2);
  for (int i = threadIdx.x; i < g.n2; i += blockDim.x) tw[i] = twg[i];
  const C* in = sticks_of<C>(t) + (int64_t)unit * g.n2 * t.S + s0;
  // the group's stick rows straight into shared memory, every copy in flight at once
  for (int i = threadIdx.x; i < cnt * g.n2; i += blockDim.x) {
    const int z = i / cnt, sl = i - z * cnt;
    tiles::async_copy(&st[sl * g.ld2 + z], &in[(int64_t)z * t.S + sl]);
  }
  tiles::async_commit();
  tiles::async_wait<0>();
  __syncthreads();
  if constexpr (N == 0) {
    fft_lines<-1>(st, cnt, LineOffStride{g.ld2}, 1, g.p2, tw);
  } else {
    fast::pass<N, -1, 1>(st, cnt, LineOffStride{fast::pitch_of<N>()}, tw);
  }
  const double s = g.inv_n;
  if (a.accumulate) {
    // Potential change: y += FFT(dV IFFT x)/N on top of a kept H x (no kinetic term).
    bool bad = false;
    if (!GAMMA) {
      const int e0 = t.grp_entry[grp], e1 = t.grp_entry[grp + 1];
      double2* y = reinterpret_cast<double2*>(a.y + (int64_t)unit * a.ldy);
      for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
        const int2 en = t.entries[e];
        const double2 h = make_double2(st[en.y].x, st[en.y].y);
        const double2 old = y[en.x];
        bad |= !finite2(old.x, old.y);
        y[en.x] = make_double2(old.x + h.x * s, old.y + h.y * s);
      }
    } else {
      const int r0 = t.grp_rep[grp], r1 = t.grp_rep[grp + 1];
      const int ca = 2 * unit;
      const bool hasb = ca + 1 < a.cols;
      double* ya = a.y + (int64_t)ca * a.ldy;
      double* yb = a.y + (int64_t)(hasb ? ca + 1 : ca) * a.ldy;
      for (int e = r0 + threadIdx.x; e < r1; e += blockDim.x) {
        const int4 rp = t.reps[e];
        const int r = rp.x;
        double2 hp = make_double2(st[rp.y].x, st[rp.y].y);
        hp.x *= s;
        hp.y *= s;
        if (r == 0) {
          bad |= !isfinite(ya[0]);
          ya[0] += hp.x;
          if (hasb) {
            bad |= !isfinite(yb[0]);
            yb[0] += hp.y;
          }
        } else {
          double2 hm = make_double2(st[rp.z].x, st[rp.z].y);
          hm.x *= s;
          hm.y *= s;
          const double ex = 0.5 * (hp.x + hm.x), ey = 0.5 * (hp.y - hm.y);
          const double ox = 0.5 * (hp.x - hm.x), oy = 0.5 * (hp.y + hm.y);
          bad |= !finite2(ya[r], ya[r + 1]);
          ya[r] += ex * kSqrt2;
          ya[r + 1] += ey * kSqrt2;
          if (hasb) {
            bad |= !finite2(yb[r], yb[r + 1]);
            yb[r] += oy * kSqrt2;
            yb[r + 1] += -ox * kSqrt2;
          }
        }
      }
    }
    if (bad) atomicOr(t.err, 1);
  } else if (!GAMMA) {
    const int e0 = t.grp_entry[grp], e1 = t.grp_entry[grp + 1];
    const double2* x = reinterpret_cast<const double2*>(a.x + (int64_t)unit * a.ldx);
    double2* y = reinterpret_cast<double2*>(a.y + (int64_t)unit * a.ldy);
#pragma unroll 4
    for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
      const int2 en = t.entries[e];
      const double2 h = make_double2(st[en.y].x, st[en.y].y);
      const double tk = t.kinetic[en.x];
      const double2 xv = x[en.x];
      y[en.x] = make_double2(h.x * s + tk * xv.x, h.y * s + tk * xv.y);
    }
  } else {
    const int r0 = t.grp_rep[grp], r1 = t.grp_rep[grp + 1];
    const int ca = 2 * unit;
    const bool hasb = ca + 1 < a.cols;
    const double* xa = a.x + (int64_t)ca * a.ldx;
    const double* xb = a.x + (int64_t)(hasb ? ca + 1 : ca) * a.ldx;
    double* ya = a.y + (int64_t)ca * a.ldy;
    double* yb = a.y + (int64_t)(hasb ? ca + 1 : ca) * a.ldy;
#pragma unroll 4
    for (int e = r0 + threadIdx.x; e < r1; e += blockDim.x) {
      const int4 rp = t.reps[e];
      const int r = rp.x;
      double2 hp = make_double2(st[rp.y].x, st[rp.y].y);
      hp.x *= s;
      hp.y *= s;
      if (r == 0) {
        const double tk = t.kinetic[0];
        ya[0] = hp.x + tk * xa[0];
        if (hasb) yb[0] = hp.y + tk * xb[0];
      } else {
        double2 hm = make_double2(st[rp.z].x, st[rp.z].y);
        hm.x *= s;
        hm.y *= s;
        // even = (hp + conj hm)/2, odd = (hp - conj hm)/2
        const double ex = 0.5 * (hp.x + hm.x), ey = 0.5 * (hp.y - hm.y);
        const double ox = 0.5 * (hp.x - hm.x), oy = 0.5 * (hp.y + hm.y);
        const double t1 = t.kinetic[r], t2 = t.kinetic[r + 1];
        ya[r] = ex * kSqrt2 + t1 * xa[r];
        ya[r + 1] = ey * kSqrt2 + t2 * xa[r + 1];
        if (hasb) {
          yb[r] = oy * kSqrt2 + t1 * xb[r];
          yb[r + 1] = -ox * kSqrt2 + t2 * xb[r + 1];
        }
      }
    }
  }
}

// ---------------------------------------------------------------- nonlocal
template <class T>
struct Ops;
template <>
struct Ops<double> {
  __device__ static double zero() { return 0.0; }
  __device__ static double cmac(double acc, double a, double b) { return fma(a, b, acc); }  // a^* b
  __device__ static double mac(double acc, double a, double b) { return fma(a, b, acc); }
  __device__ static double add(double a, double b) { return a + b; }
  __device__ static double scale(double d, double a) { return d * a; }
};
template <>
struct Ops<double2> {
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
  __device__ static double2 scale(double d, double2 a) { return make_double2(d * a.x, d * a.y); }
};

// part[ks][c][p] = sum_{rows of chunk ks} P[p][row]^* X[c][row]; tile 32 p x 32 c.
template <class T>
__global__ void __launch_bounds__(256, 2) k_project(const NlDev* __restrict__ nls, int nproj, int ksplit,
                                                    int kchunk, Batch b) {
  const int kb = blockIdx.z / ksplit, ks = blockIdx.z - kb * ksplit;
  const NlDev& nl = nls[kb];
  const CallArgs ca = resolve(b.a[kb]);
  const int cols = ca.cols, rows = nl.rows;
  if ((int)blockIdx.y * 48 >= cols) return;
  const int64_t r0 = (int64_t)ks * kchunk, r1 = min((int64_t)rows, r0 + kchunk);
  tiles::tn_tile48_mma<T>(reinterpret_cast<const T*>(nl.p), rows, reinterpret_cast<const T*>(ca.x),
                      ca.ldx / (int64_t)(sizeof(T) / sizeof(double)), blockIdx.x * 48, blockIdx.y * 48, nproj, cols,
                      r0, r1, reinterpret_cast<T*>(nl.part) + (int64_t)ks * cols * nproj, nproj);
}

// wd[c][off+i] = sum_j D[i][j] (sum_ks part[ks][c][off+j]) for one (atom, column).
template <class T>
__global__ void k_couple(const NlDev* __restrict__ nls, int nproj, int ksplit, Batch b) {
  __shared__ T w[64];
  const NlDev& nl = nls[blockIdx.z];
  const int cols = resolve(b.a[blockIdx.z]).cols;
  const int atom = blockIdx.x, c = blockIdx.y;
  if (c >= cols) return;
  const T* __restrict__ part = reinterpret_cast<const T*>(nl.part);
  T* __restrict__ wd = reinterpret_cast<T*>(nl.wd);
  const int* __restrict__ atom_off = nl.atom_off;
  const int* __restrict__ d_off = nl.d_off;
  const double* __restrict__ d = nl.d;
  const int off = atom_off[atom], cnt = atom_off[atom + 1] - off;
  const int i = threadIdx.x;
  if (i < cnt) {
    T s = Ops<T>::zero();
    for (int ks = 0; ks < ksplit; ++ks) s = Ops<T>::add(s, part[((int64_t)ks * cols + c) * nproj + off + i]);
    w[i] = s;
  }
  __syncthreads();
  if (i < cnt) {
    const double* dd = d + d_off[atom] + i * cnt;
    T s = Ops<T>::zero();
    for (int j = 0; j < cnt; ++j) s = Ops<T>::add(s, Ops<T>::scale(dd[j], w[j]));
    wd[(int64_t)c * nproj + off + i] = s;
  }
}

// y[c][row] += sum_p P[p][row] wd[c][p]; tile 64 rows x 32 columns.
template <class T>
__global__ void __launch_bounds__(256, 2) k_back(const NlDev* __restrict__ nls, int nproj, Batch b) {
  const NlDev& nl = nls[blockIdx.z];
  const CallArgs ca = resolve(b.a[blockIdx.z]);
  const int cols = ca.cols, rows = nl.rows;
  const int64_t r0 = (int64_t)blockIdx.x * 64;
  const int j0 = blockIdx.y * 64;
  if (r0 >= rows || j0 >= cols) return;
  tiles::nn_tile64_mma<T>(reinterpret_cast<const T*>(nl.p), rows, reinterpret_cast<const T*>(nl.wd), nproj,
                      reinterpret_cast<T*>(ca.y), ca.ldy / (int64_t)(sizeof(T) / sizeof(double)), rows, cols, nproj,
                      r0, j0, true);
}

// ---------------------------------------------------------------- band density
// One (z plane, chunk of units) per block: for each unit of the chunk in order, the
// plane of its inverse transform (y on the occupied x rows, x on every column) is
// built in shared memory and w |psi|^2 is added to the block's own slice of `part`
// (each thread owns the same points for every unit, so no barrier guards the sums).
// Reference: crates/dft-physics/src/distributed_complex.rs:485-547 (complex, sum in
// band order of weight |u(r)|^2 / volume), distributed_real_gamma.rs:744-785 (Gamma
// pairs: weight_a Re^2 + weight_b Im^2).
__device__ __forceinline__ void density_weights(const CallArgs& a, int gamma, const double* __restrict__ w, int unit,
                                                double* wa, double* wb) {
  if (gamma) {
    *wa = w[2 * unit];
    *wb = 2 * unit + 1 < a.cols ? w[2 * unit + 1] : 0.0;
  } else {
    *wa = *wb = w[unit];
  }
}

// Blocks of k_density_planes_fast per SM: 2 up to 45^3 planes (128 registers), 1 above,
// where the loop over units keeps more stage indices live than 128 registers hold.
template <int N>
constexpr int density_blocks_per_sm() {
  return N <= 45 ? 2 : 1;
}

// One block per (z plane, chunk of units, k point).  Per unit: the y inverse on the x
// rows holding sticks (first stage straight from the stick row), the x inverse on every
// column y (rows without sticks are zero and not loaded), then w |psi|^2 added point by
// point.  Up to 4 points per thread the sums stay in registers and the block writes its
// slice once; larger planes add into the slice in global memory unit by unit.
template <int N, bool ONE = false>
__global__ void __launch_bounds__(256, ONE ? 4 : density_blocks_per_sm<N>()) k_density_planes_fast(
    const OpTables* __restrict__ tabs, BoxGeo g, Batch b, int gamma, const double* __restrict__ w, int wstride,
    int per_chunk, double* __restrict__ part) {
  using Pl = fast::Plan<N>;
  static_assert(Pl::nst == 2, "two-stage plans");
  constexpr int R1 = Pl::radix[0], R2 = Pl::radix[1];
  constexpr int QP = (N * N + 255) / 256;
  constexpr bool REG = !ONE && QP <= 4;
  const OpTables& t = tabs[blockIdx.z];
  const CallArgs& a = b.a[blockIdx.z];
  w += (int64_t)blockIdx.z * wstride;
  const int z = blockIdx.x, chunk = blockIdx.y + blockIdx.z * gridDim.y;
  constexpr int P = fast::pitch_of<N>();
  extern __shared__ double2 sm[];
  double2* tw = sm;
  double2* pl = sm + N;
  int* rows = reinterpret_cast<int*>(pl + N * P);
  const int nx = t.nxact;
  for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = g.tw0[i];
  for (int i = threadIdx.x; i < nx; i += blockDim.x) rows[i] = t.xact[i] * P;
  double* acc = part + ((int64_t)chunk * N + z) * (N * N);
  const int u0 = blockIdx.y * per_chunk, u1 = min(a.units, u0 + per_chunk);
  double racc[REG ? QP : 1];
#pragma unroll
  for (int q = 0; q < (REG ? QP : 1); ++q) racc[q] = 0.0;
  if (u0 >= u1 && !REG)  // a k point with fewer units than the widest: its chunk adds nothing
    for (int i = threadIdx.x; i < N * N; i += blockDim.x) acc[i] = 0.0;
  __syncthreads();
  fast::StageIo<double2> io;
  io.tab = t.line_stick;
  io.xb = t.xbits;
  const int lane = threadIdx.x & 31;
  // ONE (one unit per block): no state is carried across units
  for (int unit = u0; unit < (ONE ? min(u1, u0 + 1) : u1); ++unit) {
    io.row = t.sbuf + ((int64_t)unit * N + z) * t.S;
    int first, count;
    fast::owned_block(nx, t.yper, &first, &count);
    if (count > 0) {
      fast::stage<N, R1, 1, 1, 1, fast::kInGlobal>(pl, first, count, LineOffTable{rows}, tw, lane, io);
      fast::stage<N, R2, R1, 1, 1>(pl, first, count, LineOffTable{rows}, tw, lane);
    }
    __syncthreads();
    constexpr int xper = fast::balanced_lines<N, 1, 1>(N, 8);
    fast::owned_block(N, xper, &first, &count);
    if (count > 0) {
      fast::stage<N, R1, 1, 1, P, fast::kInMask>(pl, first, count, LineOffCols{}, tw, lane, io);
      fast::stage<N, R2, R1, 1, P>(pl, first, count, LineOffCols{}, tw, lane);
    }
    __syncthreads();
    double wa, wb;
    density_weights(a, gamma, w, unit, &wa, &wb);
    if constexpr (REG) {
#pragma unroll
      for (int q = 0; q < QP; ++q) {
        const int i = threadIdx.x + 256 * q;
        if (i < N * N) {
          const int y = i / N, x = i - y * N;
          const double2 p = pl[x * P + y];
          racc[q] += wa * (p.x * p.x);
          racc[q] += wb * (p.y * p.y);
        }
      }
    } else {
      for (int i = threadIdx.x; i < N * N; i += blockDim.x) {
        const int y = i / N, x = i - y * N;
        const double2 p = pl[x * P + y];
        double d = unit == u0 ? 0.0 : acc[i];
        d += wa * (p.x * p.x);
        d += wb * (p.y * p.y);
        acc[i] = d;
      }
    }
    __syncthreads();
  }
  if constexpr (REG) {
#pragma unroll
    for (int q = 0; q < QP; ++q) {
      const int i = threadIdx.x + 256 * q;
      if (i < N * N) acc[i] = racc[q];
    }
  }
}

__global__ void __launch_bounds__(256, 1) k_density_planes(const OpTables* __restrict__ tabs, BoxGeo g, Batch b,
                                                        int gamma, const double* __restrict__ w, int wstride,
                                                        int per_chunk, double* __restrict__ part) {
  const OpTables& t = tabs[blockIdx.z];
  const CallArgs& a = b.a[blockIdx.z];
  w += (int64_t)blockIdx.z * wstride;
  const int z = blockIdx.x, chunk = blockIdx.y + blockIdx.z * gridDim.y;
  const int u0 = blockIdx.y * per_chunk, u1 = min(a.units, u0 + per_chunk);
  extern __shared__ double2 sm[];
  double2* tw0 = sm;
  double2* tw1 = tw0 + g.n0;
  double2* pl = tw1 + g.n1;
  for (int i = threadIdx.x; i < g.n0; i += blockDim.x) tw0[i] = g.tw0[i];
  for (int i = threadIdx.x; i < g.n1; i += blockDim.x) tw1[i] = g.tw1[i];
  const int np = g.n0 * g.pitch, pts = g.n0 * g.n1;
  double* acc = part + ((int64_t)chunk * g.n2 + z) * pts;
  if (u0 >= u1)
    for (int i = threadIdx.x; i < pts; i += blockDim.x) acc[i] = 0.0;
  for (int unit = u0; unit < u1; ++unit) {
    for (int i = threadIdx.x; i < np; i += blockDim.x) pl[i] = make_double2(0.0, 0.0);
    __syncthreads();
    const double2* row = t.sbuf + ((int64_t)unit * g.n2 + z) * t.S;
    for (int s = threadIdx.x; s < t.S; s += blockDim.x) pl[t.stick_plane[s]] = row[s];
    fft_lines<1>(pl, t.nxact, LineOffRows{t.xact, g.pitch}, 1, g.p1, tw1);
    fft_lines<1>(pl, g.n1, LineOffCols{}, g.pitch, g.p0, tw0);
    double wa, wb;
    density_weights(a, gamma, w, unit, &wa, &wb);
    for (int i = threadIdx.x; i < pts; i += blockDim.x) {
      const int y = i / g.n0, x = i - y * g.n0;
      const double2 p = pl[x * g.pitch + y];
      double d = unit == u0 ? 0.0 : acc[i];
      d += wa * (p.x * p.x);
      d += wb * (p.y * p.y);
      acc[i] = d;
    }
    __syncthreads();
  }
}

// ksum[k][q] = (sum_c part[k][c][q]) / volume, chunks in order (q in the partial slices'
// z, y, x order); blockIdx.y = k, so the k points' chains run side by side.
__global__ void k_density_sum_chunks(const double* __restrict__ part, int chunks, int64_t total, double volume,
                                     double* __restrict__ ksum) {
  const int k = blockIdx.y;
  const double* pk = part + (int64_t)k * chunks * total;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
#pragma unroll 8
    for (int c = 0; c < chunks; ++c) s += pk[(int64_t)c * total + q];
    ksum[(int64_t)k * total + q] = s / volume;
  }
}

// out[x][y][z] (= or +=) sum_k ksum[k][z][y n0 + x], k points added one after the other
// (the arithmetic of one call per k point accumulating into out).
__global__ void k_density_sum_k(const double* __restrict__ ksum, int nk, int n0, int n1, int n2, int accumulate,
                                double* __restrict__ out) {
  const int64_t pts = (int64_t)n0 * n1, total = pts * n2;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
    const int z = (int)(q / pts);
    const int64_t xy = q - (int64_t)z * pts;
    const int y = (int)(xy / n0), x = (int)(xy - (int64_t)y * n0);
    const int64_t p = ((int64_t)x * n1 + y) * n2 + z;
    double o = accumulate ? out[p] : 0.0;
    for (int k = 0; k < nk; ++k) {
      const double s = ksum[(int64_t)k * total + q];
      o = (k == 0 && !accumulate) ? s : o + s;
    }
    out[p] = o;
  }
}

__global__ void k_potential_transpose(const double* __restrict__ v, int n0, int n1, int n2, int vstride,
                                      double* __restrict__ vt, int* err) {
  const int64_t pts = (int64_t)n0 * n1, total = pts * n2;
  bool bad = false;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
    const int z = (int)(q / pts);
    const int64_t xy = q - z * pts;
    const int y = (int)(xy / n0), x = (int)(xy - (int64_t)y * n0);
    const double w = v[((int64_t)x * n1 + y) * n2 + z];
    bad |= !isfinite(w);
    vt[(int64_t)z * vstride + xy] = w;
  }
  if (bad) atomicOr(err, 2);
}

}  // namespace

size_t plane_smem_bytes(const BoxGeo& g) {
  const bool vs = g.n0 == g.n1 && v_in_smem(g.n0);
  return sizeof(double2) * ((size_t)g.n0 + g.n1 + (size_t)g.n0 * g.pitch) +
         (vs ? sizeof(double) * (size_t)g.n0 * g.n1 : 0) + sizeof(int) * (size_t)g.n0;
}
size_t stick_smem_bytes(const BoxGeo& g) { return sizeof(double2) * ((size_t)g.n2 + (size_t)g.sg * g.ld2); }
static size_t plane_smem_bytes_f32(const BoxGeo& g) {
  return sizeof(float2) * ((size_t)g.n0 + (size_t)g.n0 * g.pitch) +
         (v_in_smem_t<float2>(g.n0) ? sizeof(float) * (size_t)g.n0 * g.n1 : 0) + sizeof(int) * (size_t)g.n0;
}
static size_t stick_smem_bytes_f32(const BoxGeo& g) { return sizeof(float2) * ((size_t)g.n2 + (size_t)g.sg * g.ld2); }

int plane_lines_per_warp(int n0, int n1, int nlines, int warps) {
  if (n0 != n1) return 1;
  switch (n0) {
    case 25: return fast::balanced_lines<25, 1, 1>(nlines, warps);
    case 45: return fast::balanced_lines<45, 1, 1>(nlines, warps);
    case 54: return fast::balanced_lines<54, 1, 1>(nlines, warps);
    case 60: return fast::balanced_lines<60, 1, 1>(nlines, warps);
    case 72: return fast::balanced_lines<72, 1, 1>(nlines, warps);
    case 108: return fast::balanced_lines<108, 1, 1>(nlines, warps);
    default: return 1;
  }
}

bool fp32_supported(const BoxGeo& g) {
  if (g.n0 != g.n1 || g.n1 != g.n2) return false;
  switch (g.n2) {
    case 25: case 45: case 54: case 60: case 72: case 108: return true;
    default: return false;
  }
}

namespace {
struct StageScope {
  StageEvents* ev;
  int s;
  cudaStream_t st;
  StageScope(StageEvents* e, int stage, cudaStream_t stream) : ev(e), s(stage), st(stream) {
    if (ev && ev->on) cudaEventRecord(ev->ev[2 * s], st);
  }
  ~StageScope() {
    if (ev && ev->on) cudaEventRecord(ev->ev[2 * s + 1], st);
  }
};
}  // namespace

template <bool GAMMA, int N, class C>
static void local_kernels(const OpTables* tabs, const BoxGeo& g, const Batch& b, dim3 sgrid, dim3 pgrid, size_t ss,
                          size_t ps, cudaStream_t s, StageEvents* ev) {
  constexpr int st = N == 0 ? 256 : 128;
  if constexpr (N == 0 && sizeof(C) != sizeof(double2)) {
    return;  // the FP32 apply needs a compile-time plan (checked by the callers)
  } else {
    { StageScope sc(ev, 0, s); k_sticks_inverse<GAMMA, N, C><<<sgrid, st, ss, s>>>(tabs, g, b); }
    if constexpr (N == 0) {
      StageScope sc(ev, 1, s);
      k_planes<<<pgrid, 512, ps, s>>>(tabs, g, b);
    } else {
      StageScope sc(ev, 1, s);
      if (g.n0 == N && g.n1 == N)
        k_planes_fast<N, C><<<pgrid, planes_threads<N, C>(), ps, s>>>(tabs, g, b);
      else if constexpr (sizeof(C) == sizeof(double2))
        k_planes<<<pgrid, 512, ps, s>>>(tabs, g, b);
    }
    { StageScope sc(ev, 2, s); k_sticks_forward<GAMMA, N, C><<<sgrid, st, ss, s>>>(tabs, g, b); }
  }
}

template <bool GAMMA, class C>
static void local_dispatch(const OpTables* tabs, const BoxGeo& g, const Batch& b, dim3 sgrid, dim3 pgrid, size_t ss,
                           size_t ps, cudaStream_t s, StageEvents* ev) {
  switch (g.n2) {
    case 25: local_kernels<GAMMA, 25, C>(tabs, g, b, sgrid, pgrid, ss, ps, s, ev); break;
    case 45: local_kernels<GAMMA, 45, C>(tabs, g, b, sgrid, pgrid, ss, ps, s, ev); break;
    case 54: local_kernels<GAMMA, 54, C>(tabs, g, b, sgrid, pgrid, ss, ps, s, ev); break;
    case 60: local_kernels<GAMMA, 60, C>(tabs, g, b, sgrid, pgrid, ss, ps, s, ev); break;
    case 72: local_kernels<GAMMA, 72, C>(tabs, g, b, sgrid, pgrid, ss, ps, s, ev); break;
    case 108: local_kernels<GAMMA, 108, C>(tabs, g, b, sgrid, pgrid, ss, ps, s, ev); break;
    default: local_kernels<GAMMA, 0, C>(tabs, g, b, sgrid, pgrid, ss, ps, s, ev); break;
  }
}

int launch_local(const OpTables* tabs, int gamma, int max_groups, const BoxGeo& g, const Batch& b, cudaStream_t s,
                 StageEvents* ev, int fp32) {
  int max_units = 0;
  for (int k = 0; k < b.nk; ++k) max_units = max(max_units, b.a[k].units);
  if (max_units == 0 || b.nk == 0) return 0;
  const dim3 sgrid(max_groups, max_units, b.nk);
  const dim3 pgrid(max_units, g.n2, b.nk);
  if (fp32) {
    if (!fp32_supported(g)) return 0;
    const size_t ss = stick_smem_bytes_f32(g), ps = plane_smem_bytes_f32(g);
    if (gamma)
      local_dispatch<true, float2>(tabs, g, b, sgrid, pgrid, ss, ps, s, ev);
    else
      local_dispatch<false, float2>(tabs, g, b, sgrid, pgrid, ss, ps, s, ev);
    return 3;
  }
  const size_t ss = stick_smem_bytes(g), ps = plane_smem_bytes(g);
  if (gamma)
    local_dispatch<true, double2>(tabs, g, b, sgrid, pgrid, ss, ps, s, ev);
  else
    local_dispatch<false, double2>(tabs, g, b, sgrid, pgrid, ss, ps, s, ev);
  return 3;
}

// vtf[z vsf + q] = (float) vt[z vs + q], q < n0 n1.
__global__ void k_potential_float(const double* __restrict__ vt, int vs, float* __restrict__ vtf, int vsf, int plane,
                                  int n2) {
  const int64_t total = (int64_t)plane * n2;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t z = t / plane, q = t - z * plane;
    vtf[z * vsf + q] = (float)vt[z * vs + q];
  }
}

void launch_potential_float(const double* vt, const BoxGeo& g, float* vtf, cudaStream_t s) {
  const int plane = g.n0 * g.n1;
  const int64_t total = (int64_t)plane * g.n2;
  const int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 8);
  k_potential_float<<<blocks, 256, 0, s>>>(vt, g.vstride, vtf, g.vstridef, plane, g.n2);
}

size_t density_smem_bytes(const BoxGeo& g) {
  const bool fast = g.n0 == g.n1 && g.n1 == g.n2;
  return sizeof(double2) * ((size_t)g.n0 + g.n1 + (size_t)g.n0 * g.pitch) + (fast ? sizeof(int) * (size_t)g.n0 : 0);
}

template <int N>
static void density_kernels(const OpTables* tabs, int gamma, int max_groups, const BoxGeo& g, const Batch& b,
                            int max_units, const double* w, int wstride, int per_chunk, int chunks, double* part,
                            cudaStream_t s) {
  constexpr int st = N == 0 ? 256 : 128;
  const dim3 sgrid(max_groups, max_units, b.nk);
  const size_t ss = stick_smem_bytes(g), ds = density_smem_bytes(g);
  if (gamma)
    k_sticks_inverse<true, N><<<sgrid, st, ss, s>>>(tabs, g, b);
  else
    k_sticks_inverse<false, N><<<sgrid, st, ss, s>>>(tabs, g, b);
  const dim3 dgrid(g.n2, chunks, b.nk);
  if constexpr (N != 0) {
    if (g.n0 == N && g.n1 == N) {
      if (per_chunk == 1)
        k_density_planes_fast<N, true><<<dgrid, 256, ds, s>>>(tabs, g, b, gamma, w, wstride, per_chunk, part);
      else
        k_density_planes_fast<N><<<dgrid, 256, ds, s>>>(tabs, g, b, gamma, w, wstride, per_chunk, part);
      return;
    }
  }
  k_density_planes<<<dgrid, 256, ds, s>>>(tabs, g, b, gamma, w, wstride, per_chunk, part);
}

int launch_density(const OpTables* tabs, int gamma, int max_groups, const BoxGeo& g, const Batch& b,
                   const double* weights, int wstride, int per_chunk, int chunks, double* part, cudaStream_t s) {
  int max_units = 0;
  for (int k = 0; k < b.nk; ++k) max_units = max(max_units, b.a[k].units);
  if (max_units == 0 || b.nk == 0) return 0;
  switch (g.n2) {
#define BG_DENS(NN) \
  case NN: density_kernels<NN>(tabs, gamma, max_groups, g, b, max_units, weights, wstride, per_chunk, chunks, part, s); break;
    BG_DENS(25) BG_DENS(45) BG_DENS(54) BG_DENS(60) BG_DENS(72) BG_DENS(108)
#undef BG_DENS
    default: density_kernels<0>(tabs, gamma, max_groups, g, b, max_units, weights, wstride, per_chunk, chunks, part, s); break;
  }
  return 2;
}

void launch_density_reduce(const double* part, int nk, int chunks, const BoxGeo& g, double volume, int accumulate,
                           double* ksum, double* out, cudaStream_t s) {
  const int64_t total = (int64_t)g.n0 * g.n1 * g.n2;
  const int bx = (int)std::min<int64_t>((total + 255) / 256, std::max<int64_t>(1, 148 * 8 / std::max(nk, 1) + 1));
  k_density_sum_chunks<<<dim3(bx, nk), 256, 0, s>>>(part, chunks, total, volume, ksum);
  const int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 8);
  k_density_sum_k<<<blocks, 256, 0, s>>>(ksum, nk, g.n0, g.n1, g.n2, accumulate, out);
}

__global__ void k_gather_errors(int* const* __restrict__ err, int n, int* __restrict__ out) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    out[i] = *err[i];
    *err[i] = 0;
  }
}

void launch_gather_errors(int* const* err, int n, int* out, cudaStream_t s) {
  k_gather_errors<<<1, 64, 0, s>>>(err, n, out);
}

// dst[j][i] = src[i] for every destination j (blockIdx.y).
__global__ void k_broadcast(const double* __restrict__ src, int64_t n, double* const* __restrict__ dst) {
  double* d = dst[blockIdx.y];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    d[i] = src[i];
}

void launch_broadcast(const double* src, int64_t n, double* const* dst, int ndst, cudaStream_t s) {
  if (n <= 0 || ndst <= 0) return;
  const int bx = (int)std::min<int64_t>((n + 255) / 256, std::max(1, 2 * 148 / ndst + 1));
  k_broadcast<<<dim3(bx, ndst), 256, 0, s>>>(src, n, dst);
}

void launch_potential_transpose(const double* v, const BoxGeo& g, double* vt, int* err, cudaStream_t s) {
  const int64_t total = (int64_t)g.n0 * g.n1 * g.n2;
  const int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 8);
  k_potential_transpose<<<blocks, 256, 0, s>>>(v, g.n0, g.n1, g.n2, g.vstride, vt, err);
}

int launch_nonlocal(const NlDev* nl, int gamma, const NlShape& sh, int max_rows, const Batch& b, cudaStream_t s,
                    StageEvents* ev) {
  int max_cols = 0;
  for (int k = 0; k < b.nk; ++k) max_cols = max(max_cols, b.a[k].cols);
  if (sh.nproj == 0 || max_cols == 0 || b.nk == 0) return 0;
  const dim3 pg((sh.nproj + 47) / 48, (max_cols + 47) / 48, sh.ksplit * b.nk);
  const dim3 cg(sh.natoms, max_cols, b.nk);
  const dim3 bg_((max_rows + 63) / 64, (max_cols + 63) / 64, b.nk);
  const int cth = ((sh.maxch + 31) / 32) * 32;
  if (gamma) {
    {
      StageScope sc(ev, 3, s);
      k_project<double><<<pg, 256, tiles::tn48m_smem_bytes<double>(), s>>>(nl, sh.nproj, sh.ksplit, sh.kchunk, b);
    }
    { StageScope sc(ev, 4, s); k_couple<double><<<cg, cth, 0, s>>>(nl, sh.nproj, sh.ksplit, b); }
    { StageScope sc(ev, 5, s); k_back<double><<<bg_, 256, tiles::nn64m_smem_bytes<double>(), s>>>(nl, sh.nproj, b); }
  } else {
    {
      StageScope sc(ev, 3, s);
      k_project<double2><<<pg, 256, tiles::tn48m_smem_bytes<double2>(), s>>>(nl, sh.nproj, sh.ksplit, sh.kchunk, b);
    }
    { StageScope sc(ev, 4, s); k_couple<double2><<<cg, cth, 0, s>>>(nl, sh.nproj, sh.ksplit, b); }
    {
      StageScope sc(ev, 5, s);
      k_back<double2><<<bg_, 256, tiles::nn64m_smem_bytes<double2>(), s>>>(nl, sh.nproj, b);
    }
  }
  return 3;
}

}  // namespace bg

namespace bg {

// Opt every kernel with dynamic shared memory into the sizes one operator needs.
template <bool GAMMA, int N>
static void configure_one(cudaError_t& e, size_t plane_smem, size_t stick_smem) {
  auto set = [&](const void* f, size_t bytes) {
    if (e == cudaSuccess) e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  };
  auto carve = [&](const void* f) {
    if (e == cudaSuccess) e = cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  };
  set((const void*)k_sticks_inverse<GAMMA, N>, stick_smem);
  set((const void*)k_sticks_forward<GAMMA, N>, stick_smem);
  carve((const void*)k_sticks_inverse<GAMMA, N>);
  carve((const void*)k_sticks_forward<GAMMA, N>);
  if constexpr (N != 0) {
    set((const void*)k_planes_fast<N>, plane_smem);
    carve((const void*)k_planes_fast<N>);
    set((const void*)k_planes_fast<N, float2>, plane_smem);
    carve((const void*)k_planes_fast<N, float2>);
    set((const void*)k_sticks_inverse<GAMMA, N, float2>, stick_smem);
    set((const void*)k_sticks_forward<GAMMA, N, float2>, stick_smem);
    carve((const void*)k_sticks_inverse<GAMMA, N, float2>);
    carve((const void*)k_sticks_forward<GAMMA, N, float2>);
    if constexpr (GAMMA) {
      set((const void*)k_density_planes_fast<N>, plane_smem);
      carve((const void*)k_density_planes_fast<N>);
      set((const void*)k_density_planes_fast<N, true>, plane_smem);
      carve((const void*)k_density_planes_fast<N, true>);
    }
  }
}

int configure_kernels(size_t plane_smem, size_t stick_smem) {
  cudaError_t e = cudaSuccess;
  e = cudaFuncSetAttribute((const void*)k_project<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)tiles::tn48m_smem_bytes<double>());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void*)k_project<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)tiles::tn48m_smem_bytes<double2>());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void*)k_back<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)tiles::nn64m_smem_bytes<double>());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void*)k_back<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)tiles::nn64m_smem_bytes<double2>());
  if (e != cudaSuccess) return 1;
  e = cudaFuncSetAttribute((const void*)k_planes, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)plane_smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void*)k_density_planes, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)plane_smem);
  configure_one<true, 0>(e, plane_smem, stick_smem);
  configure_one<false, 0>(e, plane_smem, stick_smem);
  configure_one<true, 25>(e, plane_smem, stick_smem);
  configure_one<false, 25>(e, plane_smem, stick_smem);
  configure_one<true, 45>(e, plane_smem, stick_smem);
  configure_one<false, 45>(e, plane_smem, stick_smem);
  configure_one<true, 54>(e, plane_smem, stick_smem);
  configure_one<false, 54>(e, plane_smem, stick_smem);
  configure_one<true, 60>(e, plane_smem, stick_smem);
  configure_one<false, 60>(e, plane_smem, stick_smem);
  configure_one<true, 72>(e, plane_smem, stick_smem);
  configure_one<false, 72>(e, plane_smem, stick_smem);
  configure_one<true, 108>(e, plane_smem, stick_smem);
  configure_one<false, 108>(e, plane_smem, stick_smem);
  return e == cudaSuccess ? 0 : 1;
}

// Descriptors of the tensor-core nonlocal products of every operator of a batch:
// [k] P^H x into the projection buffer, [nk + k] y += P wd, P from the operator's
// split panels.  One thread per operator.
__global__ void k_nl_tc_descs(const NlDev* __restrict__ nls, int nproj, Batch b, tc::ZDesc* __restrict__ out) {
  const int k = threadIdx.x;
  if (k >= b.nk) return;
  const NlDev& nl = nls[k];
  const CallArgs ca = resolve(b.a[k]);
  const int cols = ca.cols;
  const double2* p = reinterpret_cast<const double2*>(nl.p);
  out[k] = tc::ZDesc{p,     reinterpret_cast<const double2*>(ca.x), reinterpret_cast<double2*>(nl.part), nl.rows,
                     ca.ldx / 2, nproj, cols > 0 ? nproj : 0, cols, nl.rows, tc::kStore, nl.p_tn, nl.kt_tn};
  out[b.nk + k] = tc::ZDesc{p, reinterpret_cast<const double2*>(nl.wd), reinterpret_cast<double2*>(ca.y), nl.rows,
                            nproj, ca.ldy / 2, cols > 0 ? nl.rows : 0, cols, nproj, tc::kAdd, nl.p_nn, nl.kt_nn};
}

void TcNl::release() {
  cudaFree(desc);
  cudaFree(work);
  cudaFree(err);
  desc = nullptr;
  work = nullptr;
  err = nullptr;
  work_bytes = 0;
}

int ensure_nonlocal_tc(TcNl* t, int nk, int nproj, int max_cols, int max_rows) {
  cudaError_t e = tc::prepare_zgemm();
  if (e != cudaSuccess) return 1;
  if (!t->desc && cudaMalloc(&t->desc, sizeof(tc::ZDesc) * 2 * kMaxBatch) != cudaSuccess) return 1;
  if (!t->err) {
    if (cudaMalloc(&t->err, sizeof(int)) != cudaSuccess) return 1;
    if (cudaMemset(t->err, 0, sizeof(int)) != cudaSuccess) return 1;
  }
  t->ksplit = tc::tn_ksplit_tuned(nk, nproj, max_cols, max_rows);
  // the projection and the back-projection run one after the other on one stream and
  // share the workspace
  const size_t need = std::max(tc::workspace_bytes(tc::kTN, nk, nproj, max_cols, max_rows, t->ksplit, true),
                               tc::workspace_bytes(tc::kNN, nk, max_rows, max_cols, nproj, 1, true));
  if (need > t->work_bytes) {
    cudaFree(t->work);
    t->work = nullptr;
    t->work_bytes = 0;
    if (cudaMalloc(&t->work, need) != cudaSuccess) return 1;
    t->work_bytes = need;
  }
  return 0;
}

int launch_nonlocal_tc(const NlDev* nl, const NlShape& sh, int max_rows, int max_cols, const Batch& b, TcNl* t,
                       cudaStream_t s, StageEvents* ev) {
  if (sh.nproj == 0 || max_cols == 0 || b.nk == 0) return 0;
  tc::ZDesc* d = static_cast<tc::ZDesc*>(t->desc);
  int launches = 1;
  k_nl_tc_descs<<<1, kMaxBatch, 0, s>>>(nl, sh.nproj, b, d);
  {
    StageScope sc(ev, 3, s);
    launches += tc::launch_zgemm(tc::kTN, d, b.nk, sh.nproj, max_cols, max_rows, t->ksplit, true, t->work, t->err, s);
  }
  {
    StageScope sc(ev, 4, s);
    const dim3 cg(sh.natoms, max_cols, b.nk);
    k_couple<double2><<<cg, ((sh.maxch + 31) / 32) * 32, 0, s>>>(nl, sh.nproj, 1, b);
    launches += 1;
  }
  {
    StageScope sc(ev, 5, s);
    launches += tc::launch_zgemm(tc::kNN, d + b.nk, b.nk, max_rows, max_cols, sh.nproj, 1, true, t->work, t->err, s);
  }
  return launches;
}

}  // namespace bg
