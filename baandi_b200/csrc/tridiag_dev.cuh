// Real symmetric tridiagonal eigensolver for one thread block (the control block of the
// batched Davidson): all eigenvalues by Sturm-sequence multisection, eigenvectors by
// inverse iteration with modified Gram-Schmidt inside clusters of close eigenvalues.
// This is the published bisection / inverse-iteration scheme (Sturm counts with the
// pivmin safeguard, Gershgorin brackets, shifted LU with partial pivoting, the cluster
// tolerance 1e-3 |T|_1 and the 10 eps |T|_1 separation of shifts inside a cluster), laid
// out for a GPU block: every eigenvalue is bracketed by a group of lanes that each count
// two shifts per round; every eigenvector is one thread's inverse iteration, and the
// vectors of a cluster are then orthonormalised in order (Gram-Schmidt twice) by one
// warp, its lanes over the rows.  Shifts inside a run of eigenvalues closer than 10 eps |T|_1 are spread by that
// amount and the start vectors differ, so the iterates of a near-degenerate cluster span
// its invariant subspace; components outside it shrink by (shift error / gap)^2 over the
// two solves.
//
// Input: d (m diagonal entries) and e (m - 1 couplings, e[i] between i and i+1, any sign)
// in shared memory.  Output: wu[j] and eigenvector j in Z, entry r at Z[r ldz + j]
// (row-major, so that the threads of different clusters touch adjacent words), j < m,
// eigenpairs in ascending order inside each unreduced block (blocks in row order); Z is
// zero outside each vector's block.  Scratch: e2 (m doubles, shared), starts and clusters (m + 1 ints
// each, shared), lu1 and lu2 (lu*_doubles each, best in shared memory: 4 m doubles for
// every eigenvector computed at the same time, so together at least 4 m).
#pragma once

namespace bg {
namespace tri {

constexpr double kUlp = 2.220446049250313e-16;
constexpr double kSafeMin = 2.2250738585072014e-308;
constexpr int kMaxRounds = 100;
constexpr int kInverseIterations = 5;
constexpr int kExtraIterations = 1;   // after the growth criterion is met

// 2^-e(v) for the binary exponent e(v) of a finite nonzero v (bits of an IEEE double):
// an exact power of two that brings |v| into [1, 2).
__device__ __forceinline__ double exponent_scale(double v) {
  const long long bits = __double_as_longlong(v);
  const long long e = (bits >> 52) & 0x7ff;                 // biased exponent, 1..2046 here
  return __longlong_as_double((long long)(2046 - e) << 52);  // 2^(1023 - e)
}

// Sturm counts of the eigenvalues below each of the C shifts x[c] in block [s, s + n):
// the sign changes along the leading principal minors p_0 = 1, p_1 = d_s - x,
// p_r+1 = (d_s+r - x) p_r - e_s+r-1^2 p_r-1 (a zero minor takes the sign opposite to its
// predecessor).  The recurrence has one fused multiply-add on its dependent chain (no
// division) and the C shifts run interleaved.  After every 8 steps each pair of minors is
// rescaled by an exact power of two (from the larger one's exponent bits, no branch): 8
// steps grow a minor by at most (2 |T|_1)^8, far inside the exponent range for the
// reduced matrices here (|T|_1 well below 2^60).
template <int C>
__device__ __forceinline__ void sturm(const double* d, const double* e2, int s, int n, const double (&x)[C],
                                      int (&cnt)[C]) {
  double p[C], q[C];
  bool sg[C];
#pragma unroll
  for (int c = 0; c < C; ++c) {
    p[c] = d[s] - x[c];
    q[c] = 1.0;
    sg[c] = p[c] <= 0.0;
    cnt[c] = sg[c];
  }
  auto step = [&](int i) {
    const double di = d[i], ei = e2[i - 1];
#pragma unroll
    for (int c = 0; c < C; ++c) {
      const double r = fma(di - x[c], p[c], -ei * q[c]);
      q[c] = p[c];
      p[c] = r;
      const bool ng = r == 0.0 ? !sg[c] : r < 0.0;
      cnt[c] += ng != sg[c];
      sg[c] = ng;
    }
  };
  int i = s + 1;
  for (; i + 8 <= s + n; i += 8) {
#pragma unroll
    for (int u = 0; u < 8; ++u) step(i + u);
#pragma unroll
    for (int c = 0; c < C; ++c) {
      const double big = fmax(fabs(p[c]), fabs(q[c]));
      const double f = exponent_scale(big);
      p[c] *= f;
      q[c] *= f;
    }
  }
  for (; i < s + n; ++i) step(i);
}

// Block of eigenvalue j (blocks listed by their first rows in starts[0..nb]).
__device__ __forceinline__ int block_of(const int* starts, int nb, int j) {
  int b = 0;
  while (b + 1 < nb && starts[b + 1] <= j) ++b;
  return b;
}

// Gershgorin interval of block [s, s + n), widened by the rounding of the counts, and
// its 1-norm.
__device__ __forceinline__ void gershgorin(const double* d, const double* e, int s, int n, double pivmin,
                                           double* gl, double* gu, double* onenrm) {
  double lo = 1e300, hi = -1e300, nrm = 0.0;
  for (int i = s; i < s + n; ++i) {
    const double r = (i > s ? fabs(e[i - 1]) : 0.0) + (i + 1 < s + n ? fabs(e[i]) : 0.0);
    lo = fmin(lo, d[i] - r);
    hi = fmax(hi, d[i] + r);
    nrm = fmax(nrm, fabs(d[i]) + r);
  }
  const double tn = fmax(fabs(lo), fabs(hi));
  const double pad = 2.0 * kUlp * tn * n + 2.0 * pivmin;
  *gl = lo - pad;
  *gu = hi + pad;
  *onenrm = nrm;
}

// Deterministic start vector entry in (-1, 1) for row r of eigenvector j.
__device__ __forceinline__ double start_entry(int j, int r) {
  unsigned h = 2654435761u * (unsigned)(j + 1) ^ (2246822519u * (unsigned)(r + 7));
  h ^= h >> 15;
  h *= 2246822519u;
  h ^= h >> 13;
  h *= 3266489917u;
  h ^= h >> 16;
  return 2.0 * ((double)h * (1.0 / 4294967296.0)) - 1.0;
}

template <int NT>
__device__ void eig(int m, const double* __restrict__ d, const double* __restrict__ e, double* e2, double* wu,
                    int* starts, int* clusters, double* Z, int ldz, double* __restrict__ lu1, int lu1_doubles,
                    double* __restrict__ lu2, int lu2_doubles, int* sh) {
  // 1. splits where a coupling is negligible against its neighbours; squared couplings
  if (threadIdx.x == 0) {
    int nb = 0;
    starts[nb++] = 0;
    for (int i = 0; i + 1 < m; ++i) {
      if (fabs(e[i]) <= kUlp * (fabs(d[i]) + fabs(d[i + 1]))) {
        e2[i] = 0.0;
        starts[nb++] = i + 1;
      } else {
        e2[i] = e[i] * e[i];
      }
    }
    starts[nb] = m;
    sh[0] = nb;
  }
  for (int t = threadIdx.x; t < m * m; t += NT) Z[(t % m) + (size_t)(t / m) * ldz] = 0.0;
  __syncthreads();
  const int nb = sh[0];
  double e2max = 1.0;
  for (int i = 0; i + 1 < m; ++i) e2max = fmax(e2max, e2[i]);
  const double pivmin = kSafeMin * e2max;

  // 2. eigenvalues: G lanes per eigenvalue, each counting kShifts shifts per round;
  //    located to 2 eps max(|lo|, |hi|) + eps |T_b|_1.  A lane's Sturm step issues about
  //    7 instructions per shift and the warps of one group are issue-bound, so the time of
  //    a bracket goes as kShifts / log(G kShifts + 1): two shifts per lane beat four and
  //    eight (35, 50 and 78 us per 34 x 34 solve on one B200)
  constexpr int kShifts = 2;
  int G = 1;
  while (G < 32 && 2 * G * m <= NT) G *= 2;
  const int NG = NT / G, gid = threadIdx.x / G, lig = threadIdx.x % G;
  const unsigned gmask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << ((threadIdx.x & 31) & ~(G - 1)));
  for (int j0 = 0; j0 < m; j0 += NG) {
    const int j = j0 + gid;
    const bool act = j < m;
    int s = 0, n = 1, i = 0;
    double lo = 0.0, hi = 0.0, nrm = 0.0;
    if (act) {
      const int b = block_of(starts, nb, j);
      s = starts[b];
      n = starts[b + 1] - s;
      i = j - s;
      gershgorin(d, e, s, n, pivmin, &lo, &hi, &nrm);
    }
    bool done = !act;
    const int K = kShifts * G;
    const double atol = kUlp * nrm + 2.0 * pivmin;
    for (int it = 0; it < kMaxRounds; ++it) {
      if (!done) {
        if (hi - lo <= 2.0 * kUlp * fmax(fabs(lo), fabs(hi)) + atol) {
          done = true;
        } else {
          const double h = (hi - lo) / (K + 1);
          const int r0 = kShifts * lig;
          double xs[kShifts];
          int cs[kShifts];
#pragma unroll
          for (int c = 0; c < kShifts; ++c) xs[c] = lo + (r0 + c + 1) * h;
          sturm<kShifts>(d, e2, s, n, xs, cs);
          int rf = K;
#pragma unroll
          for (int c = kShifts - 1; c >= 0; --c)
            if (cs[c] > i) rf = r0 + c;
          for (int o = G >> 1; o > 0; o >>= 1) rf = min(rf, __shfl_xor_sync(gmask, rf, o));
          const double nlo = rf > 0 ? lo + rf * h : lo;
          const double nhi = rf < K ? lo + (rf + 1) * h : hi;
          lo = nlo;
          hi = nhi;
        }
      }
      if (__all_sync(0xffffffffu, done)) break;
    }
    if (act && lig == 0) wu[j] = 0.5 * (lo + hi);
  }
  __syncthreads();

  // 3. clusters: consecutive eigenvalues of one block closer than 1e-3 |T_b|_1
  if (threadIdx.x == 0) {
    int nc = 0;
    for (int b = 0; b < nb; ++b) {
      const int s = starts[b], n = starts[b + 1] - s;
      double gl, gu, nrm;
      gershgorin(d, e, s, n, pivmin, &gl, &gu, &nrm);
      const double ortol = 1e-3 * nrm;
      clusters[nc++] = s;
      for (int j = s + 1; j < s + n; ++j)
        if (wu[j] - wu[j - 1] > ortol) clusters[nc++] = j;
    }
    clusters[nc] = m;
    sh[1] = nc;
  }
  __syncthreads();
  const int nc = sh[1];

  // 4. eigenvectors: one thread per eigenvector, inverse iteration on its block.  A
  //    thread's LU strips (reciprocal pivots, first and second superdiagonals of U,
  //    multipliers) hold 4 m doubles, so at most (lu1 + lu2) / (4 m) threads work at a
  //    time.  A row swap at elimination step r < n - 2 leaves a nonzero second
  //    superdiagonal (the couplings inside a block are nonzero); the swap at step n - 2 is
  //    kept apart.
  const int P1 = lu1_doubles / (4 * m), P2 = lu2_doubles / (4 * m);
  const int P = max(1, min(NT, P1 + P2));
  for (int j = threadIdx.x; j < m && threadIdx.x < P; j += P) {
    const int b = block_of(starts, nb, j);
    const int s = starts[b], n = starts[b + 1] - s;
    if (n == 1) {
      Z[(size_t)s * ldz + j] = 1.0;
      continue;
    }
    double gl, gu, onenrm;
    gershgorin(d, e, s, n, pivmin, &gl, &gu, &onenrm);
    const double pertol = 10.0 * kUlp * onenrm, tiny = kUlp * onenrm;
    const double dtpcrt = sqrt(0.1 / n);
    const bool first_region = (int)threadIdx.x < P1;
    const int ps = first_region ? P1 : P2;
    double* ur = first_region ? lu1 + threadIdx.x : lu2 + (threadIdx.x - P1);
    double* u1 = ur + (size_t)m * ps;
    double* u2 = u1 + (size_t)m * ps;
    double* lm = u2 + (size_t)m * ps;
    // shift: spread by pertol along a run of eigenvalues closer than pertol
    int jr = j;
    while (jr > s && wu[jr] - wu[jr - 1] < pertol) --jr;
    const double x = wu[j] + (j - jr) * pertol;
    // LU with partial pivoting of T_b - x I; pivots below eps |T|_1 are raised to it
    // (the solve then grows along the eigenvector) and kept as reciprocals
    double ai = d[s] - x, bi = e[s], ulast = 0.0;
    bool last_swap = false;
    for (int r = 0; r + 1 < n; ++r) {
      const double ci = e[s + r], an = d[s + r + 1] - x, bn = r + 2 < n ? e[s + r + 1] : 0.0;
      double l, piv;
      if (fabs(ai) >= fabs(ci)) {
        l = ai != 0.0 ? ci / ai : 0.0;
        piv = ai;
        u1[(size_t)r * ps] = bi;
        u2[(size_t)r * ps] = 0.0;
        ai = an - l * bi;
        bi = bn;
      } else {
        l = ai / ci;
        piv = ci;
        u1[(size_t)r * ps] = an;
        u2[(size_t)r * ps] = bn;
        ai = bi - l * an;
        bi = -l * bn;
        if (r + 2 == n) last_swap = true;
      }
      if (fabs(piv) < tiny) piv = piv < 0.0 ? -tiny : tiny;
      ur[(size_t)r * ps] = 1.0 / piv;
      lm[(size_t)r * ps] = l;
    }
    if (fabs(ai) < tiny) ai = ai < 0.0 ? -tiny : tiny;
    ulast = fabs(ai);
    ur[(size_t)(n - 1) * ps] = 1.0 / ai;
    // z(r) below stands for Z[(s + r) ldz + j]
    double* zc = Z + (size_t)s * ldz + j;
    auto z = [&](int r) -> double& { return zc[(size_t)r * ldz]; };
    double asum = 0.0;
    for (int r = 0; r < n; ++r) {
      const double v = start_entry(j, r);
      z(r) = v;
      asum += fabs(v);
    }
    int checks = 0;
    for (int its = 0; its < kInverseIterations; ++its) {
      const double scl = n * onenrm * fmax(kUlp, ulast) / asum;
      // L^-1 P (scaled right-hand side); the running entry rides in a register
      double zr = z(0) * scl;
      for (int r = 0; r + 1 < n; ++r) {
        double zn = z(r + 1) * scl;
        const bool sw = r + 2 < n ? u2[(size_t)r * ps] != 0.0 : last_swap;
        if (sw) {
          const double t = zr;
          zr = zn;
          zn = t;
        }
        z(r) = zr;
        zr = zn - lm[(size_t)r * ps] * zr;
      }
      // U^-1; the two previous entries ride in registers
      double z1 = zr * ur[(size_t)(n - 1) * ps];
      z(n - 1) = z1;
      double z0 = (z(n - 2) - u1[(size_t)(n - 2) * ps] * z1) * ur[(size_t)(n - 2) * ps];
      z(n - 2) = z0;
      double zmax = fmax(fabs(z1), fabs(z0));
      asum = fabs(z1) + fabs(z0);
      for (int r = n - 3; r >= 0; --r) {
        const double v = (z(r) - u1[(size_t)r * ps] * z0 - u2[(size_t)r * ps] * z1) * ur[(size_t)r * ps];
        z(r) = v;
        z1 = z0;
        z0 = v;
        zmax = fmax(zmax, fabs(v));
        asum += fabs(v);
      }
      if (zmax >= dtpcrt && ++checks > kExtraIterations) break;
    }
    double nn = 0.0;
    for (int r = 0; r < n; ++r) nn += z(r) * z(r);
    const double inv = 1.0 / sqrt(nn);
    for (int r = 0; r < n; ++r) z(r) *= inv;
  }
  __syncthreads();

  // 5. each cluster's vectors orthonormalised in order (Gram-Schmidt, twice), then the
  //    sign: the largest entry of every vector positive.  One warp per cluster, the lanes
  //    over the rows; dot products and norms are warp sums.
  {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int cidx = warp; cidx < nc; cidx += NT / 32) {
      const int ja = clusters[cidx], jb = clusters[cidx + 1];
      const int b = block_of(starts, nb, ja);
      const int s = starts[b], n = starts[b + 1] - s;
      const double* zb = Z + (size_t)s * ldz;
      for (int j = ja; j < jb; ++j) {
        double* zc = Z + (size_t)s * ldz + j;
        for (int pass = 0; pass < 2 && j > ja; ++pass) {
          for (int q = ja; q < j; ++q) {
            double dot = 0.0;
            for (int r = lane; r < n; r += 32) dot = fma(zc[(size_t)r * ldz], zb[(size_t)r * ldz + q], dot);
            for (int o = 16; o > 0; o >>= 1) dot += __shfl_xor_sync(0xffffffffu, dot, o);
            for (int r = lane; r < n; r += 32) zc[(size_t)r * ldz] = fma(-dot, zb[(size_t)r * ldz + q], zc[(size_t)r * ldz]);
            __syncwarp();
          }
          double nn = 0.0;
          for (int r = lane; r < n; r += 32) nn = fma(zc[(size_t)r * ldz], zc[(size_t)r * ldz], nn);
          for (int o = 16; o > 0; o >>= 1) nn += __shfl_xor_sync(0xffffffffu, nn, o);
          const double inv = 1.0 / sqrt(nn);
          for (int r = lane; r < n; r += 32) zc[(size_t)r * ldz] *= inv;
          __syncwarp();
        }
        // sign: the first entry of largest magnitude positive
        double big = -1.0;
        int at = n;
        for (int r = lane; r < n; r += 32) {
          const double v = fabs(zc[(size_t)r * ldz]);
          if (v > big) {
            big = v;
            at = r;
          }
        }
        for (int o = 16; o > 0; o >>= 1) {
          const double ob = __shfl_xor_sync(0xffffffffu, big, o);
          const int oa = __shfl_xor_sync(0xffffffffu, at, o);
          if (ob > big || (ob == big && oa < at)) {
            big = ob;
            at = oa;
          }
        }
        const bool neg = zc[(size_t)at * ldz] < 0.0;
        __syncwarp();
        if (neg)
          for (int r = lane; r < n; r += 32) zc[(size_t)r * ldz] = -zc[(size_t)r * ldz];
        __syncwarp();
      }
    }
  }
  __syncthreads();
}

}  // namespace tri
}  // namespace bg
