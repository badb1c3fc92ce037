// Real symmetric tridiagonal eigensolver for one thread block (the control block of the
// batched Davidson): all eigenvalues by Sturm-sequence multisection, eigenvectors by
// inverse iteration with modified Gram-Schmidt inside clusters of close eigenvalues.
// This is the published bisection / inverse-iteration scheme (Sturm counts with the
// pivmin safeguard, Gershgorin brackets, shifted LU with partial pivoting, the cluster
// tolerance 1e-3 |T|_1 and the 10 eps |T|_1 separation of shifts inside a cluster), laid
// out for a GPU block: every eigenvalue is bracketed by a group of lanes that each count
// two shifts per round, and every cluster of eigenvectors is one thread's serial work.
//
// Input: d (m diagonal entries) and e (m - 1 couplings, e[i] between i and i+1, any sign)
// in shared memory.  Output: wu[j] and eigenvector j in Z, entry r at Z[r ldz + j]
// (row-major, so that the threads of different clusters touch adjacent words), j < m,
// eigenpairs in ascending order inside each unreduced block (blocks in row order); Z is
// zero outside each vector's block.  Scratch: e2 (m doubles, shared), starts and clusters (m + 1 ints
// each, shared), lu (5 m NT doubles, global, one strip per thread).
#pragma once

namespace bg {
namespace tri {

constexpr double kUlp = 2.220446049250313e-16;
constexpr double kSafeMin = 2.2250738585072014e-308;
constexpr int kMaxRounds = 100;
constexpr int kInverseIterations = 5;
constexpr int kExtraIterations = 1;   // after the growth criterion is met

// Sturm counts of the eigenvalues below xa and below xb of block [s, s + n): the sign
// changes along the leading principal minors p_0 = 1, p_1 = d_s - x,
// p_r+1 = (d_s+r - x) p_r - e_s+r-1^2 p_r-1 (a zero minor takes the sign opposite to its
// predecessor).  The recurrence has one fused multiply-add on its dependent chain (no
// division), two shifts run interleaved, and a pair of minors is rescaled by an exact
// power of two when it leaves [2^-500, 2^500].
__device__ __forceinline__ void sturm2(const double* d, const double* e2, int s, int n, double xa, double xb,
                                       int* ca, int* cb) {
  double pa = d[s] - xa, pb = d[s] - xb, qa = 1.0, qb = 1.0;  // p_r, p_r-1
  bool sa = pa <= 0.0, sb = pb <= 0.0;                         // sign bit of p_r (zero: opposite of p_0 > 0)
  int a = sa, b = sb;
  for (int i = s + 1; i < s + n; ++i) {
    const double di = d[i], ei = e2[i - 1];
    const double ra = fma(di - xa, pa, -ei * qa);
    const double rb = fma(di - xb, pb, -ei * qb);
    qa = pa;
    pa = ra;
    qb = pb;
    pb = rb;
    const bool na = pa == 0.0 ? !sa : pa < 0.0;
    const bool nb = pb == 0.0 ? !sb : pb < 0.0;
    a += na != sa;
    b += nb != sb;
    sa = na;
    sb = nb;
    if (!(fabs(pa) < 0x1p500) || fabs(pa) < 0x1p-500) {
      const int ex = ilogb(pa == 0.0 ? qa : pa);
      pa = scalbn(pa, -ex);
      qa = scalbn(qa, -ex);
    }
    if (!(fabs(pb) < 0x1p500) || fabs(pb) < 0x1p-500) {
      const int ex = ilogb(pb == 0.0 ? qb : pb);
      pb = scalbn(pb, -ex);
      qb = scalbn(qb, -ex);
    }
  }
  *ca = a;
  *cb = b;
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
                    int* starts, int* clusters, double* Z, int ldz, double* __restrict__ lu, int* sh) {
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

  // 2. eigenvalues: G lanes per eigenvalue, each counting two shifts per round
  int G = 1;
  while (G < 32 && 2 * G * m <= NT) G *= 2;
  const int NG = NT / G, gid = threadIdx.x / G, lig = threadIdx.x % G;
  const unsigned gmask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << ((threadIdx.x & 31) & ~(G - 1)));
  for (int j0 = 0; j0 < m; j0 += NG) {
    const int j = j0 + gid;
    const bool act = j < m;
    int s = 0, n = 1, i = 0;
    double lo = 0.0, hi = 0.0, nrm;
    if (act) {
      const int b = block_of(starts, nb, j);
      s = starts[b];
      n = starts[b + 1] - s;
      i = j - s;
      gershgorin(d, e, s, n, pivmin, &lo, &hi, &nrm);
    }
    bool done = !act;
    const int K = 2 * G;
    for (int it = 0; it < kMaxRounds; ++it) {
      if (!done) {
        if (hi - lo <= 2.0 * kUlp * fmax(fabs(lo), fabs(hi)) + 2.0 * pivmin) {
          done = true;
        } else {
          const double h = (hi - lo) / (K + 1);
          const int r0 = 2 * lig;
          int c0, c1;
          sturm2(d, e2, s, n, lo + (r0 + 1) * h, lo + (r0 + 2) * h, &c0, &c1);
          int rf = c0 > i ? r0 : (c1 > i ? r0 + 1 : K);
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

  // 4. eigenvectors: one cluster per thread, inverse iteration on its block
  for (int cidx = threadIdx.x; cidx < nc; cidx += NT) {
    const int ja = clusters[cidx], jb = clusters[cidx + 1];
    const int b = block_of(starts, nb, ja);
    const int s = starts[b], n = starts[b + 1] - s;
    if (n == 1) {
      Z[(size_t)s * ldz + ja] = 1.0;
      continue;
    }
    double gl, gu, onenrm;
    gershgorin(d, e, s, n, pivmin, &gl, &gu, &onenrm);
    const double pertol = 10.0 * kUlp * onenrm, tiny = kUlp * onenrm;
    const double dtpcrt = sqrt(0.1 / n);
    // this thread's strips: U diagonal, first and second superdiagonals, multipliers, pivots
    double* u0 = lu + threadIdx.x;
    double* u1 = u0 + (size_t)m * NT;
    double* u2 = u1 + (size_t)m * NT;
    double* lm = u2 + (size_t)m * NT;
    double* pv = lm + (size_t)m * NT;
    double xprev = 0.0;
    for (int j = ja; j < jb; ++j) {
      double x = wu[j];
      if (j > ja && x - xprev < pertol) x = xprev + pertol;
      xprev = x;
      // LU with partial pivoting of T_b - x I
      double ai = d[s] - x, bi = e[s];
      for (int r = 0; r + 1 < n; ++r) {
        const double ci = e[s + r], an = d[s + r + 1] - x, bn = r + 2 < n ? e[s + r + 1] : 0.0;
        double l;
        if (fabs(ai) >= fabs(ci)) {
          l = ai != 0.0 ? ci / ai : 0.0;
          u0[(size_t)r * NT] = ai;
          u1[(size_t)r * NT] = bi;
          u2[(size_t)r * NT] = 0.0;
          pv[(size_t)r * NT] = 0.0;
          ai = an - l * bi;
          bi = bn;
        } else {
          l = ai / ci;
          u0[(size_t)r * NT] = ci;
          u1[(size_t)r * NT] = an;
          u2[(size_t)r * NT] = bn;
          pv[(size_t)r * NT] = 1.0;
          ai = bi - l * an;
          bi = -l * bn;
        }
        lm[(size_t)r * NT] = l;
      }
      u0[(size_t)(n - 1) * NT] = ai;
      // pivots below eps |T|_1 raised to it (the solve then grows along the eigenvector);
      // the back substitution multiplies by their reciprocals
      double ulast = 0.0;
      for (int r = 0; r < n; ++r) {
        double u = u0[(size_t)r * NT];
        if (fabs(u) < tiny) u = u < 0.0 ? -tiny : tiny;
        if (r == n - 1) ulast = fabs(u);
        u0[(size_t)r * NT] = 1.0 / u;
      }
      // z(r) below stands for Z[(s + r) ldz + j]
      double* zc = Z + (size_t)s * ldz + j;
      auto z = [&](int r) -> double& { return zc[(size_t)r * ldz]; };
      for (int r = 0; r < n; ++r) z(r) = start_entry(j, r);
      int checks = 0;
      for (int its = 0; its < kInverseIterations; ++its) {
        double asum = 0.0;
        for (int r = 0; r < n; ++r) asum += fabs(z(r));
        const double scl = n * onenrm * fmax(kUlp, ulast) / asum;
        for (int r = 0; r < n; ++r) z(r) *= scl;
        // L^-1 P
        for (int r = 0; r + 1 < n; ++r) {
          if (pv[(size_t)r * NT] != 0.0) {
            const double t = z(r);
            z(r) = z(r + 1);
            z(r + 1) = t;
          }
          z(r + 1) -= lm[(size_t)r * NT] * z(r);
        }
        // U^-1 (u0 holds the reciprocal pivots); the two previous entries ride in registers
        double z1 = z(n - 1) * u0[(size_t)(n - 1) * NT];
        z(n - 1) = z1;
        double z0 = (z(n - 2) - u1[(size_t)(n - 2) * NT] * z1) * u0[(size_t)(n - 2) * NT];
        z(n - 2) = z0;
        for (int r = n - 3; r >= 0; --r) {
          const double zr = (z(r) - u1[(size_t)r * NT] * z0 - u2[(size_t)r * NT] * z1) * u0[(size_t)r * NT];
          z(r) = zr;
          z1 = z0;
          z0 = zr;
        }
        // against the cluster's earlier vectors
        for (int jj = ja; jj < j; ++jj) {
          const double* y = Z + (size_t)s * ldz + jj;
          double dot = 0.0;
          for (int r = 0; r < n; ++r) dot += z(r) * y[(size_t)r * ldz];
          for (int r = 0; r < n; ++r) z(r) -= dot * y[(size_t)r * ldz];
        }
        double zmax = 0.0;
        for (int r = 0; r < n; ++r) zmax = fmax(zmax, fabs(z(r)));
        if (zmax >= dtpcrt && ++checks > kExtraIterations) break;
      }
      double nn = 0.0, big = 0.0, sgn = 1.0;
      for (int r = 0; r < n; ++r) {
        nn += z(r) * z(r);
        if (fabs(z(r)) > big) {
          big = fabs(z(r));
          sgn = z(r) < 0.0 ? -1.0 : 1.0;
        }
      }
      const double inv = sgn / sqrt(nn);
      for (int r = 0; r < n; ++r) z(r) *= inv;
    }
  }
  __syncthreads();
}

}  // namespace tri
}  // namespace bg
