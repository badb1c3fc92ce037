// Compile-time line FFTs for the grid lengths of the benchmark cells (FP64 or FP32 complex).
//
// A pass transforms L lines held in shared memory.  Each warp owns a contiguous block
// of lines and carries it through every radix stage alone, separated only by
// __syncwarp, so the block meets at a barrier once per pass instead of once per stage.
// Each stage is the in-place Stockham decimation-in-time step of fft_dev.cuh (element
// j + t N/R of butterfly j in, (j / Ns) Ns R + j mod Ns + u Ns out) with every index a
// constant expression.  A stage runs in rounds of whole lines (32 / (N/R) lines per
// round, one butterfly per lane): a round loads its butterflies' inputs, __syncwarp,
// stores the outputs in place, so a lane holds only R values.  Radices 2, 3, 4, 5, 6,
// 8, 9 and 12; the 6-, 8-, 9- and 12-point DFTs are Cooley-Tukey splits (2x3, 2x4,
// 3x3, 3x4) done in registers.
//
// Twiddles w^(t k N/(Ns R)) are powers of one entry of the length-N table
// exp(+2 pi i q/N) in shared memory (conjugated for the forward sign).
#pragma once
#include "fft_dev.cuh"

namespace bg {
namespace fast {

// --------------------------------------------------------------------- plans
template <int N>
struct Plan {
  static constexpr bool ok = false;
};
#define BG_PLAN(NN, ...)                                    \
  template <>                                               \
  struct Plan<NN> {                                         \
    static constexpr bool ok = true;                        \
    static constexpr int radix[] = {__VA_ARGS__};           \
    static constexpr int nst = sizeof(radix) / sizeof(int); \
  };
BG_PLAN(25, 5, 5)
BG_PLAN(45, 5, 9)
BG_PLAN(54, 6, 9)
BG_PLAN(60, 12, 5)
BG_PLAN(72, 8, 9)
BG_PLAN(108, 12, 9)
#undef BG_PLAN

// --------------------------------------------------------------------- butterflies
// C = double2 or float2; constants are rounded to the element's precision.
template <int SIGN, class C>
__device__ __forceinline__ C w_mul(C a, RealOf<C> c, RealOf<C> s) {
  // a * (c + i SIGN s)
  const RealOf<C> ss = SIGN > 0 ? s : -s;
  return mkc<C>(a.x * c - a.y * ss, a.x * ss + a.y * c);
}

template <int R, int SIGN, class C>
struct Dft;

template <int SIGN, class C>
struct Dft<2, SIGN, C> {
  __device__ __forceinline__ static void run(C* v) {
    const C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};
template <int SIGN, class C>
struct Dft<3, SIGN, C> {
  __device__ __forceinline__ static void run(C* v) {
    using T = RealOf<C>;
    const T h = T(0.8660254037844386), half = T(0.5);
    const C t1 = cadd(v[1], v[2]);
    const C t2 = mkc<C>(v[0].x - half * t1.x, v[0].y - half * t1.y);
    const C t3 = irot<SIGN>(cscale(csub(v[1], v[2]), h));
    v[0] = cadd(v[0], t1);
    v[1] = cadd(t2, t3);
    v[2] = csub(t2, t3);
  }
};
template <int SIGN, class C>
struct Dft<4, SIGN, C> {
  __device__ __forceinline__ static void run(C* v) {
    const C a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
    const C c = cadd(v[1], v[3]), d = irot<SIGN>(csub(v[1], v[3]));
    v[0] = cadd(a, c);
    v[2] = csub(a, c);
    v[1] = cadd(b, d);
    v[3] = csub(b, d);
  }
};
template <int SIGN, class C>
struct Dft<5, SIGN, C> {
  __device__ __forceinline__ static void run(C* v) {
    using T = RealOf<C>;
    const T c1 = T(0.30901699437494745), c2 = T(-0.8090169943749475);
    const T s1 = T(0.9510565162951535), s2 = T(0.5877852522924731);
    const C p1 = cadd(v[1], v[4]), m1 = csub(v[1], v[4]);
    const C p2 = cadd(v[2], v[3]), m2 = csub(v[2], v[3]);
    const C a1 = mkc<C>(v[0].x + c1 * p1.x + c2 * p2.x, v[0].y + c1 * p1.y + c2 * p2.y);
    const C a2 = mkc<C>(v[0].x + c2 * p1.x + c1 * p2.x, v[0].y + c2 * p1.y + c1 * p2.y);
    const C b1 = irot<SIGN>(mkc<C>(s1 * m1.x + s2 * m2.x, s1 * m1.y + s2 * m2.y));
    const C b2 = irot<SIGN>(mkc<C>(s2 * m1.x - s1 * m2.x, s2 * m1.y - s1 * m2.y));
    v[0] = cadd(v[0], cadd(p1, p2));
    v[1] = cadd(a1, b1);
    v[4] = csub(a1, b1);
    v[2] = cadd(a2, b2);
    v[3] = csub(a2, b2);
  }
};
// 6 = 3 x 2: a = DFT3(v0, v2, v4), b = DFT3(v1, v3, v5); X[u] = a[u] + w6^u b[u],
// X[u+3] = a[u] - w6^u b[u].
template <int SIGN, class C>
struct Dft<6, SIGN, C> {
  __device__ __forceinline__ static void run(C* v) {
    using T = RealOf<C>;
    C a[3] = {v[0], v[2], v[4]}, b[3] = {v[1], v[3], v[5]};
    Dft<3, SIGN, C>::run(a);
    Dft<3, SIGN, C>::run(b);
    const T h = T(0.8660254037844386);
    const C b1 = w_mul<SIGN>(b[1], T(0.5), h);
    const C b2 = w_mul<SIGN>(b[2], T(-0.5), h);
    v[0] = cadd(a[0], b[0]);
    v[3] = csub(a[0], b[0]);
    v[1] = cadd(a[1], b1);
    v[4] = csub(a[1], b1);
    v[2] = cadd(a[2], b2);
    v[5] = csub(a[2], b2);
  }
};
// 8 = 4 x 2: a = DFT4(evens), b = DFT4(odds); X[u] = a[u] + w8^u b[u], X[u+4] = a[u] - w8^u b[u].
template <int SIGN, class C>
struct Dft<8, SIGN, C> {
  __device__ __forceinline__ static void run(C* v) {
    using T = RealOf<C>;
    C a[4] = {v[0], v[2], v[4], v[6]}, b[4] = {v[1], v[3], v[5], v[7]};
    Dft<4, SIGN, C>::run(a);
    Dft<4, SIGN, C>::run(b);
    const T r = T(0.7071067811865476);
    const C b1 = w_mul<SIGN>(b[1], r, r);
    const C b2 = irot<SIGN>(b[2]);
    const C b3 = w_mul<SIGN>(b[3], -r, r);
    v[0] = cadd(a[0], b[0]);
    v[4] = csub(a[0], b[0]);
    v[1] = cadd(a[1], b1);
    v[5] = csub(a[1], b1);
    v[2] = cadd(a[2], b2);
    v[6] = csub(a[2], b2);
    v[3] = cadd(a[3], b3);
    v[7] = csub(a[3], b3);
  }
};
// 9 = 3 x 3: a_m = DFT3(v_m, v_{m+3}, v_{m+6}); b_m[k1] = a_m[k1] w9^(m k1);
// X[k1 + 3 k2] = DFT3 over m of b_m[k1].
template <int SIGN, class C>
struct Dft<9, SIGN, C> {
  __device__ __forceinline__ static void run(C* v) {
    using T = RealOf<C>;
    C a0[3] = {v[0], v[3], v[6]}, a1[3] = {v[1], v[4], v[7]}, a2[3] = {v[2], v[5], v[8]};
    Dft<3, SIGN, C>::run(a0);
    Dft<3, SIGN, C>::run(a1);
    Dft<3, SIGN, C>::run(a2);
    const T c1 = T(0.766044443118978), s1 = T(0.6427876096865394);    // 2 pi/9
    const T c2 = T(0.17364817766693036), s2 = T(0.984807753012208);   // 4 pi/9
    const T c4 = T(-0.9396926207859084), s4 = T(0.3420201433256687);  // 8 pi/9
    a1[1] = w_mul<SIGN>(a1[1], c1, s1);
    a1[2] = w_mul<SIGN>(a1[2], c2, s2);
    a2[1] = w_mul<SIGN>(a2[1], c2, s2);
    a2[2] = w_mul<SIGN>(a2[2], c4, s4);
#pragma unroll
    for (int k1 = 0; k1 < 3; ++k1) {
      C t[3] = {a0[k1], a1[k1], a2[k1]};
      Dft<3, SIGN, C>::run(t);
      v[k1] = t[0];
      v[k1 + 3] = t[1];
      v[k1 + 6] = t[2];
    }
  }
};

// 12 = 3 x 4: a_m = DFT4(v_m, v_{m+3}, v_{m+6}, v_{m+9}); b_m[k1] = a_m[k1] w12^(m k1);
// X[k1 + 4 k2] = DFT3 over m of b_m[k1].
template <int SIGN, class C>
struct Dft<12, SIGN, C> {
  __device__ __forceinline__ static void run(C* v) {
    using T = RealOf<C>;
    C a0[4] = {v[0], v[3], v[6], v[9]}, a1[4] = {v[1], v[4], v[7], v[10]}, a2[4] = {v[2], v[5], v[8], v[11]};
    Dft<4, SIGN, C>::run(a0);
    Dft<4, SIGN, C>::run(a1);
    Dft<4, SIGN, C>::run(a2);
    const T h = T(0.8660254037844386), half = T(0.5);
    a1[1] = w_mul<SIGN>(a1[1], h, half);   // w12^1
    a1[2] = w_mul<SIGN>(a1[2], half, h);   // w12^2
    a1[3] = irot<SIGN>(a1[3]);             // w12^3
    a2[1] = w_mul<SIGN>(a2[1], half, h);   // w12^2
    a2[2] = w_mul<SIGN>(a2[2], -half, h);  // w12^4
    a2[3] = mkc<C>(-a2[3].x, -a2[3].y);    // w12^6
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
      C t[3] = {a0[k1], a1[k1], a2[k1]};
      Dft<3, SIGN, C>::run(t);
      v[k1] = t[0];
      v[k1 + 4] = t[1];
      v[k1 + 8] = t[2];
    }
  }
};

// --------------------------------------------------------------------- stages
// Lane index read with a volatile instruction: the per-lane butterfly indices of a stage
// are then recomputed where the stage runs instead of being hoisted out of an enclosing
// loop (a persistent kernel would otherwise keep every stage's indices live in registers).
__device__ __forceinline__ int lane_id() {
  int l;
  asm volatile("mov.u32 %0, %%laneid;" : "=r"(l));
  return l;
}

// Where a stage reads its inputs and writes its outputs.  IO = 0: the warp's lines in
// shared memory (base + off(line) + element ES).  Bits of IO change one side:
//   kInGlobal   inputs of line i from the stick row in global memory: element e is
//               row[tab[i N + e]], zero where tab holds -1 (no stick at that position)
//   kOutGlobal  outputs of line i to row[tab[i N + e]], dropped where tab holds -1
//   kInMask     inputs at elements whose bit is clear in xb are zero (not loaded)
//   kOutMask    outputs at elements whose bit is clear in xb are not stored
constexpr int kInGlobal = 1, kOutGlobal = 2, kInMask = 4, kOutMask = 8;
template <class C>
struct StageIo {
  const int* tab = nullptr;
  C* row = nullptr;
  const unsigned* xb = nullptr;  // element bits (4 words, N <= 128)
};

__device__ __forceinline__ unsigned xbit(const unsigned* xb, int e) { return (__ldg(xb + (e >> 5)) >> (e & 31)) & 1u; }

// Stage (R, NS) on lines first .. first+count-1 of this warp; ES = element stride.
// A lane's butterfly index j, its twiddle and its element masks are the same in every
// round, so they are set up once before the rounds.
template <int N, int R, int NS, int SIGN, int ES, int IO = 0, class Off, class C>
__device__ __forceinline__ void stage(C* base, int first, int count, Off off, const C* __restrict__ tw, int lane,
                                      const StageIo<C>& io = StageIo<C>{}) {
  constexpr int SPAN = N / R;
  constexpr int STEP = N / (NS * R);
  constexpr int K = (SPAN + 31) / 32;                 // butterflies per lane when a line exceeds a warp
  constexpr int LPR = SPAN <= 32 ? 32 / SPAN : 1;     // whole lines per round
  lane = lane_id();
  int jj[K], li[K], oo[K];
  unsigned tin[K], tout[K];
  int kk[K];
#pragma unroll
  for (int q = 0; q < K; ++q) {
    const int slot = lane + 32 * q;
    li[q] = K == 1 ? slot / SPAN : 0;
    jj[q] = K == 1 ? slot - li[q] * SPAN : slot;
    if (K == 1 ? li[q] >= LPR : jj[q] >= SPAN) li[q] = 1 << 20;  // idle lane
    const int j = jj[q] < SPAN ? jj[q] : 0;
    const int k = NS > 1 ? j % NS : 0;
    oo[q] = (NS > 1 ? (j / NS) * NS * R : j * R) + k;
    kk[q] = k * STEP;
    tin[q] = tout[q] = 0u;
    if constexpr ((IO & kInMask) != 0) {
#pragma unroll
      for (int t = 0; t < R; ++t) tin[q] |= xbit(io.xb, j + t * SPAN) << t;
    }
    if constexpr ((IO & kOutMask) != 0) {
#pragma unroll
      for (int u = 0; u < R; ++u) tout[q] |= xbit(io.xb, oo[q] + u * NS) << u;
    }
  }
  for (int r0 = 0; r0 < count; r0 += LPR) {
    C v[K][R];
    int lo[K], ln[K];
#pragma unroll
    for (int q = 0; q < K; ++q) {
      const bool act = r0 + li[q] < count;
      ln[q] = first + r0 + li[q];
      lo[q] = act ? off(ln[q]) : -1;
      if (act) {
        if constexpr ((IO & kInGlobal) != 0) {
          int sidx[R];
#pragma unroll
          for (int t = 0; t < R; ++t) sidx[t] = __ldg(io.tab + ln[q] * N + jj[q] + t * SPAN);
#pragma unroll
          for (int t = 0; t < R; ++t) v[q][t] = sidx[t] >= 0 ? io.row[sidx[t]] : mkc<C>(0.0, 0.0);
        } else {
#pragma unroll
          for (int t = 0; t < R; ++t)
            v[q][t] = ((IO & kInMask) == 0 || ((tin[q] >> t) & 1u)) ? base[lo[q] + (jj[q] + t * SPAN) * ES]
                                                                   : mkc<C>(0.0, 0.0);
        }
      }
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < K; ++q) {
      if (lo[q] >= 0) {
        if (NS > 1) {
          // w^(t k STEP) as powers of one table entry: one shared-memory load per
          // butterfly instead of R - 1 (relative error grows by about one ulp per power)
          C w1 = tw[kk[q]];
          if (SIGN < 0) w1.y = -w1.y;
          C x = w1;
#pragma unroll
          for (int t = 1; t < R; ++t) {
            v[q][t] = cmul(v[q][t], x);
            if (t + 1 < R) x = cmul(x, w1);
          }
        }
        Dft<R, SIGN, C>::run(v[q]);
        if constexpr ((IO & kOutGlobal) != 0) {
#pragma unroll
          for (int u = 0; u < R; ++u) {
            const int sx = __ldg(io.tab + ln[q] * N + oo[q] + u * NS);
            if (sx >= 0) io.row[sx] = v[q][u];
          }
        } else {
#pragma unroll
          for (int u = 0; u < R; ++u)
            if ((IO & kOutMask) == 0 || ((tout[q] >> u) & 1u)) base[lo[q] + (oo[q] + u * NS) * ES] = v[q][u];
        }
      }
    }
    __syncwarp();
  }
}

template <int N, int SIGN, int ES, int S, int NS, class Off, class C>
__device__ __forceinline__ void stages_from(C* base, int first, int count, Off off, const C* __restrict__ tw,
                                            int lane) {
  using P = Plan<N>;
  if constexpr (S < P::nst) {
    constexpr int R = P::radix[S];
    stage<N, R, NS, SIGN, ES>(base, first, count, off, tw, lane);
    stages_from<N, SIGN, ES, S + 1, NS * R>(base, first, count, off, tw, lane);
  }
}

// Every stage of lines first .. first+count-1 (one warp; ends with __syncwarp).
template <int N, int SIGN, int ES, class Off, class C>
__device__ __forceinline__ void group(C* base, int first, int count, Off off, const C* __restrict__ tw, int lane) {
  stages_from<N, SIGN, ES, 0, 1>(base, first, count, off, tw, lane);
}

// Inverse transform, x w(element), forward transform of this warp's lines for a
// two-stage plan (R1, R2), with the middle in registers: the inverse's last stage
// (radix R2, span R1) leaves butterfly j holding elements j + u R1 (u < R2) in natural
// order, exactly the inputs of the first stage of a forward transform run with the
// plan reversed (R2, R1).  So that butterfly multiplies by w, runs the forward radix-R2
// DFT and stores once; shared memory sees load, store, load, store, load, store per
// element instead of ten accesses.  w(line, x) is read through `wgt`.  MASK: only the
// elements whose bit is set in io.xb are nonzero on input and wanted on output.
template <int N, int ES, bool MASK = false, class Off, class W, class C>
__device__ __forceinline__ void inverse_weight_forward(C* base, int first, int count, Off off,
                                                       const C* __restrict__ tw, W wgt, int lane,
                                                       const StageIo<C>& io = StageIo<C>{}) {
  using P = Plan<N>;
  static_assert(P::nst == 2, "two-stage plans only");
  constexpr int R1 = P::radix[0];
  constexpr int R2 = P::radix[1];
  stage<N, R1, 1, 1, ES, MASK ? kInMask : 0>(base, first, count, off, tw, lane, io);
  constexpr int SPAN = N / R2;  // == R1
  static_assert(SPAN <= 32, "one butterfly per lane");
  constexpr int LPR = 32 / SPAN;
  lane = lane_id();
  const int li = lane / SPAN;
  const int j = lane - li * SPAN;
  const bool lane_ok = li < LPR;
  const C w1 = tw[j];  // w^(t k N/(R1 R2)) with k = j, as powers of w^j
  for (int r0 = 0; r0 < count; r0 += LPR) {
    C v[R2];
    const bool act = lane_ok && r0 + li < count;
    const int line = first + r0 + li;
    const int lo = act ? off(line) : 0;
    if (act) {
#pragma unroll
      for (int t = 0; t < R2; ++t) v[t] = base[lo + (j + t * SPAN) * ES];
    }
    __syncwarp();
    if (act) {
      {
        C x = w1;
#pragma unroll
        for (int t = 1; t < R2; ++t) {
          v[t] = cmul(v[t], x);
          if (t + 1 < R2) x = cmul(x, w1);
        }
      }
      Dft<R2, 1, C>::run(v);
#pragma unroll
      for (int u = 0; u < R2; ++u) {
        const RealOf<C> w = wgt(line, j + u * R1);
        v[u].x *= w;
        v[u].y *= w;
      }
      Dft<R2, -1, C>::run(v);
#pragma unroll
      for (int u = 0; u < R2; ++u) base[lo + (j * R2 + u) * ES] = v[u];
    }
    __syncwarp();
  }
  // forward: remaining stage of the reversed plan, radix R1 after span R2
  stage<N, R1, R2, -1, ES, MASK ? kOutMask : 0>(base, first, count, off, tw, lane, io);
}

// Lines of a pass owned by this warp: a contiguous block of ceil(L / warps).
__device__ __forceinline__ void owned_lines(int nlines, int* first, int* count) {
  const int nw = blockDim.x >> 5, warp = threadIdx.x >> 5;
  const int per = (nlines + nw - 1) / nw;
  *first = min(nlines, warp * per);
  *count = min(nlines, *first + per) - *first;
}

// Whole lines per round of a radix-R stage on lines of N (one butterfly per lane).
__host__ __device__ constexpr int lines_per_round(int N, int R) { return N / R <= 32 ? 32 / (N / R) : 1; }

// Lines per warp for a pass of a two-stage plan whose radix-R1 round loop runs A times
// and whose span-R1 round loop (the radix-R2 stage, or the fused middle of
// inverse_weight_forward) runs B times, LA and LB whole lines per round; warps own
// contiguous blocks of that many lines.  A round issues the same instructions whether its
// lines fill the warp or not, so the count is chosen from ceil(L / warps) upwards to
// minimise the rounds all warps run together, with the busiest warp running no more rounds
// than at ceil(L / warps).  27 lines of 45 on 8 warps: blocks of 6,6,6,6,3 lines run 14
// rounds of the two stages, blocks of 4,..,4,3 run 20.  Evaluated at compile time or on
// the host: the search is too long to repeat in every block.
__host__ __device__ constexpr int balanced_lines(int LA, int LB, int A, int B, int nlines, int nw) {
  if (nlines <= 0) return 1;
  const int base = (nlines + nw - 1) / nw;
  int best = base, best_total = 0, limit = 0;
  for (int per = base; per <= nlines && per < base + LA * LB; ++per) {
    int total = 0, worst = 0;
    for (int f = 0; f < nlines; f += per) {
      const int c = per < nlines - f ? per : nlines - f;
      const int r = A * ((c + LA - 1) / LA) + B * ((c + LB - 1) / LB);
      total += r;
      worst = worst > r ? worst : r;
    }
    if (per == base) {
      best_total = total;
      limit = worst;
    } else if (worst <= limit && total < best_total) {
      best = per;
      best_total = total;
    }
  }
  return best;
}
template <int N, int A, int B>
__host__ __device__ constexpr int balanced_lines(int nlines, int nw) {
  return balanced_lines(lines_per_round(N, Plan<N>::radix[0]), lines_per_round(N, Plan<N>::radix[1]), A, B, nlines,
                        nw);
}

// This warp's block of `per` lines of a pass over nlines lines.
__device__ __forceinline__ void owned_block(int nlines, int per, int* first, int* count) {
  const int warp = threadIdx.x >> 5;
  *first = min(nlines, warp * per);
  *count = min(nlines, *first + per) - *first;
}

// A whole pass over nlines lines; ends with __syncthreads.
template <int N, int SIGN, int ES, class Off, class C>
__device__ __forceinline__ void pass(C* base, int nlines, Off off, const C* __restrict__ tw) {
  int first, count;
  owned_lines(nlines, &first, &count);
  if (count > 0) group<N, SIGN, ES>(base, first, count, off, tw, threadIdx.x & 31);
  __syncthreads();
}

// Row pitch of a shared-memory plane of N x N: odd, so that a column line (stride
// pitch) and a row line both touch distinct banks in every 8-lane phase.
template <int N>
__host__ __device__ constexpr int pitch_of() {
  return N | 1;
}

}  // namespace fast
}  // namespace bg
