// Reduced problem of the batched Davidson on many thread blocks, for capacities beyond a
// single control block (the Gamma-only supercells: capacity 2 x bands = 320 and 960).
//
// The algebra is that of the control kernel (kset_davidson.cu: chol_extend, eigen, heev),
// crates/dft-numerics/src/linalg.rs:234-444 (bordered Cholesky, A = L^-1 H_r L^-H,
// Hermitian eigensolver, C = L^-H Y) and crates/dft-solvers/src/lean_davidson.rs:62-70
// (pivot rule), laid out over the whole GPU:
//   * triangular solves: eight right-hand sides per block, staged in shared memory, the
//     factor's columns streamed from L2 once per block (column sweep);
//   * the new diagonal block of the bordered Cholesky factor: S22 - L21 L21^H by 16 x 16
//     tiles, then a panel factorisation (32 columns; the panel by one block with the pivot
//     rule, the rows below and the trailing lower triangle by every block) in one
//     cooperative launch;
//   * Householder tridiagonalisation: one cooperative launch, every block owning columns
//     of the trailing matrix (matrix-vector product and rank-2 update), one grid barrier
//     per reflector;
//   * tridiagonal eigenpairs: Sturm bisection by one warp per eigenvalue, inverse
//     iteration by one thread per eigenvector, Gram-Schmidt inside clusters of close
//     eigenvalues by one warp per cluster;
//   * back-transformation: the stored reflectors applied to diag(s) Z, a warp per column,
//     then the back solve with L^H.
// Requests come from the control kernel (Ctl::wc_* and Ctl::we_m); every kernel here
// returns at once for a k point without one, so the launches sit in the captured
// iteration graph at fixed shapes.  Grid barriers spin a bounded number of times and
// then record kWErrBarrier and return (cooperative launches make every block resident,
// so that does not happen in a healthy run).
#pragma once

namespace bg {
namespace dv {
namespace wide {

constexpr int kT = 256;                 // threads per block
constexpr int kSolveCols = 8;           // right-hand sides per block of a triangular solve
constexpr int kPanel = 32;              // Cholesky panel width
constexpr int kTile = 16;               // tiles of the border product
constexpr double kWideOrtol = 1e-6;     // cluster gap relative to the block's 1-norm
constexpr unsigned kSpinLimit = 1u << 24;
constexpr int kMaxCap = 1152;           // the Householder kernel's columns fit in shared memory

enum : int { kWErrNonfinite = 1, kWErrBarrier = 2, kWErrPivot = 4 };
enum : int { kSolveBorder = 0, kSolveLeft, kSolveRight, kSolveBack };

// All blocks of a cooperative launch meet here; false once any barrier has given up.
// Arrival by an acquire-release add on bar[0]; the last arrival resets it and releases the
// generation word bar[1], on which the others spin (acquire loads, bounded).
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ bool grid_sync(unsigned* bar, int* err) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    if (*(volatile int*)err & kWErrBarrier) {
      ok = 0;
    } else {
      const unsigned gen = ld_acquire_u32(bar + 1);
      __threadfence();
      unsigned arrived;
      asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], 1;" : "=r"(arrived) : "l"(bar) : "memory");
      if (arrived == gridDim.x - 1) {
        asm volatile("st.relaxed.gpu.global.u32 [%0], 0;" ::"l"(bar) : "memory");
        asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(bar + 1), "r"(gen + 1) : "memory");
      } else {
        unsigned spins = 0;
        while (ld_acquire_u32(bar + 1) == gen) {
          if (++spins > kSpinLimit) {
            atomicOr(err, kWErrBarrier);
            ok = 0;
            break;
          }
          if (spins > 256) __nanosleep(32);
        }
      }
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Loads that bypass L1 (data written by other blocks of a cooperative launch since the
// last barrier must not come from a stale L1 line).
__device__ __forceinline__ double ldcg(const double* p) { return __ldcg(p); }
__device__ __forceinline__ double2 ldcg(const double2* p) { return __ldcg(p); }

template <class D>
__device__ __forceinline__ D warp_sum_d(D v) {
  for (int o = 16; o > 0; o >>= 1) v = Cx<D>::add(v, Cx<D>::shfl_xor(v, o));
  return v;
}

__device__ __forceinline__ double warp_sum_r(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ------------------------------------------------------------------ triangular solves
// WHICH: kSolveBorder  T = L11^-1 S[0:m0, m0:m1], written as L[m0:m1, 0:m0] = T^H
//        kSolveLeft    Y = L^-1 H_r                      (m columns)
//        kSolveRight   A = L^-1 Y^H                      (= L^-1 H_r L^-H)
//        kSolveBack    C = L^-H Y   (L^H from LT)
// blockIdx.x = group of kSolveCols columns, blockIdx.y = k point.
template <class D, int WHICH>
__global__ void __launch_bounds__(kT) k_w_trsm(const Bufs<D>* __restrict__ bufs, const Ctl* __restrict__ ctl, int cap) {
  using X = Cx<D>;
  const int k = blockIdx.y;
  const Bufs<D> b = bufs[k];
  const Ctl c = ctl[k];
  int m, ncols, col0 = 0;
  if (WHICH == kSolveBorder) {
    if (c.status != 0 || c.wc_m1 <= c.wc_m0 || c.wc_m0 == 0) return;
    m = c.wc_m0;
    ncols = c.wc_m1 - c.wc_m0;
    col0 = c.wc_m0;
  } else {
    if (c.status != 0 || c.we_m == 0 || *(volatile int*)b.werr != 0) return;
    m = c.we_m;
    ncols = m;
  }
  const int j0 = blockIdx.x * kSolveCols;
  if (j0 >= ncols) return;
  const int nc = min(kSolveCols, ncols - j0);
  extern __shared__ __align__(16) unsigned char w_sm[];
  D* y = reinterpret_cast<D*>(w_sm);                        // [kSolveCols][cap]
  double* rd = reinterpret_cast<double*>(y + (size_t)kSolveCols * cap);
  const D* L = WHICH == kSolveBack ? b.LT : b.L;
  for (int t = threadIdx.x; t < nc * m; t += kT) {
    const int j = t / m, r = t - j * m;
    const int cj = col0 + j0 + j;
    D v;
    if (WHICH == kSolveBorder) v = b.S[r + (size_t)cj * cap];
    else if (WHICH == kSolveLeft) v = b.Hr[r + (size_t)cj * cap];
    else if (WHICH == kSolveRight) v = X::conj(b.Y[cj + (size_t)r * cap]);
    else v = b.Y[r + (size_t)cj * cap];
    y[(size_t)j * cap + r] = v;
  }
  for (int r = threadIdx.x; r < m; r += kT) rd[r] = 1.0 / X::real(L[r + (size_t)r * cap]);
  __syncthreads();
  // Every thread owns the rows r = tid + kRows i; the factor's next column for those rows is
  // loaded one step ahead, so its latency hides behind the current step.
  constexpr int kRows = (kMaxCap + kT - 1) / kT;
  D cur[kRows], nxt[kRows];
  const int first = WHICH != kSolveBack ? 0 : m - 1;
#pragma unroll
  for (int i = 0; i < kRows; ++i) {
    const int r = threadIdx.x + i * kT;
    cur[i] = r < m ? L[r + (size_t)first * cap] : X::zero();
  }
  if (WHICH != kSolveBack) {
    for (int p = 0; p < m; ++p) {
      if (p + 1 < m) {
#pragma unroll
        for (int i = 0; i < kRows; ++i) {
          const int r = threadIdx.x + i * kT;
          nxt[i] = (r < m && r > p + 1) ? L[r + (size_t)(p + 1) * cap] : X::zero();
        }
      }
      if ((int)threadIdx.x < nc) y[(size_t)threadIdx.x * cap + p] = X::scale(rd[p], y[(size_t)threadIdx.x * cap + p]);
      __syncthreads();
#pragma unroll
      for (int i = 0; i < kRows; ++i) {
        const int r = threadIdx.x + i * kT;
        if (r > p && r < m)
          for (int j = 0; j < nc; ++j)
            y[(size_t)j * cap + r] = X::sub(y[(size_t)j * cap + r], X::mul(cur[i], y[(size_t)j * cap + p]));
        cur[i] = nxt[i];
      }
      __syncthreads();
    }
  } else {
    for (int p = m - 1; p >= 0; --p) {
      if (p > 0) {
#pragma unroll
        for (int i = 0; i < kRows; ++i) {
          const int r = threadIdx.x + i * kT;
          nxt[i] = r < p - 1 ? L[r + (size_t)(p - 1) * cap] : X::zero();   // LT column p - 1
        }
      }
      if ((int)threadIdx.x < nc) y[(size_t)threadIdx.x * cap + p] = X::scale(rd[p], y[(size_t)threadIdx.x * cap + p]);
      __syncthreads();
#pragma unroll
      for (int i = 0; i < kRows; ++i) {
        const int r = threadIdx.x + i * kT;
        if (r < p)
          for (int j = 0; j < nc; ++j)
            y[(size_t)j * cap + r] = X::sub(y[(size_t)j * cap + r], X::mul(cur[i], y[(size_t)j * cap + p]));
        cur[i] = nxt[i];
      }
      __syncthreads();
    }
  }
  for (int t = threadIdx.x; t < nc * m; t += kT) {
    const int j = t / m, r = t - j * m;
    const int cj = col0 + j0 + j;
    const D v = y[(size_t)j * cap + r];
    if (WHICH == kSolveBorder) b.L[cj + (size_t)r * cap] = X::conj(v);
    else if (WHICH == kSolveLeft) b.Y[r + (size_t)cj * cap] = v;
    else if (WHICH == kSolveRight) b.A[r + (size_t)cj * cap] = v;
    else b.C[r + (size_t)cj * cap] = v;
  }
}

inline size_t trsm_smem(int cap, size_t dsize) { return (size_t)kSolveCols * cap * dsize + (size_t)cap * sizeof(double); }

// ------------------------------------------------------------------ bordered Cholesky
// L[m0:m1, m0:m1] (lower) = S22 - L21 L21^H, zero above the diagonal; 16 x 16 tiles.
template <class D>
__global__ void __launch_bounds__(kTile* kTile) k_w_border(const Bufs<D>* __restrict__ bufs, const Ctl* __restrict__ ctl,
                                                          int cap) {
  using X = Cx<D>;
  const int k = blockIdx.y;
  const Ctl c = ctl[k];
  if (c.status != 0 || c.wc_m1 <= c.wc_m0) return;
  const Bufs<D> b = bufs[k];
  const int m0 = c.wc_m0, nr = c.wc_m1 - c.wc_m0;
  const int tiles = (nr + kTile - 1) / kTile;
  if ((int)blockIdx.x >= tiles * tiles) return;
  const int ti = blockIdx.x % tiles, tj = blockIdx.x / tiles;
  if (tj > ti) {  // strictly above the diagonal: zeros
    const int i = m0 + ti * kTile + threadIdx.x % kTile, j = m0 + tj * kTile + threadIdx.x / kTile;
    if (i < c.wc_m1 && j < c.wc_m1) b.L[i + (size_t)j * cap] = X::zero();
    return;
  }
  __shared__ D a[kTile][kTile + 1], bt[kTile][kTile + 1];
  const int tx = threadIdx.x % kTile, ty = threadIdx.x / kTile;
  const int i = m0 + ti * kTile + tx, j = m0 + tj * kTile + ty;
  D acc = X::zero();
  for (int p0 = 0; p0 < m0; p0 += kTile) {
    // a[q][x] = L[i0 + x][p0 + q], bt[q][y] = L[j0 + y][p0 + q]
    {
      const int q = ty, p = p0 + q;
      const int ia = m0 + ti * kTile + tx, jb = m0 + tj * kTile + tx;
      a[q][tx] = (p < m0 && ia < c.wc_m1) ? b.L[ia + (size_t)p * cap] : X::zero();
      bt[q][tx] = (p < m0 && jb < c.wc_m1) ? b.L[jb + (size_t)p * cap] : X::zero();
    }
    __syncthreads();
#pragma unroll 4
    for (int q = 0; q < kTile; ++q) acc = X::add(acc, X::mul(a[q][tx], X::conj(bt[q][ty])));
    __syncthreads();
  }
  if (i < c.wc_m1 && j < c.wc_m1) b.L[i + (size_t)j * cap] = j <= i ? X::sub(b.S[i + (size_t)j * cap], acc) : X::zero();
}

// Factor the new diagonal block in place (panels of kPanel columns), the pivot rule on
// every column: squared pivot over the overlap diagonal >= eps / 1e-12.  Cooperative.
template <class D>
__global__ void __launch_bounds__(kT) k_w_chol(const Bufs<D>* __restrict__ bufs, const Ctl* __restrict__ ctl, int nk,
                                               int cap, unsigned* bar) {
  using X = Cx<D>;
  __shared__ D blk[kPanel][kPanel + 1];
  __shared__ int s_fail;
  const int gtid = blockIdx.x * kT + threadIdx.x, gthreads = gridDim.x * kT;
  for (int k = 0; k < nk; ++k) {
    const Ctl c = ctl[k];
    if (c.status != 0 || c.wc_m1 <= c.wc_m0) continue;
    const Bufs<D> b = bufs[k];
    const int m0 = c.wc_m0, m1 = c.wc_m1;
    for (int t = gtid; t < m0 * (m1 - m0); t += gthreads)  // above the new block
      b.L[t % m0 + (size_t)(m0 + t / m0) * cap] = X::zero();
    for (int p0 = m0; p0 < m1; p0 += kPanel) {
      const int nb = min(kPanel, m1 - p0);
      if (blockIdx.x == 0) {
        for (int t = threadIdx.x; t < nb * nb; t += kT) {
          const int i = t % nb, j = t / nb;
          blk[i][j] = j <= i ? ldcg(b.L + (p0 + i) + (size_t)(p0 + j) * cap) : X::zero();
        }
        if (threadIdx.x == 0) s_fail = 0;
        __syncthreads();
        for (int j = 0; j < nb; ++j) {
          const double dj = X::real(blk[j][j]);
          const double ratio = dj / X::real(b.S[(p0 + j) + (size_t)(p0 + j) * cap]);
          if (!(ratio >= kPivotRatioMin) || !isfinite(ratio)) {
            if (threadIdx.x == 0) s_fail = 1;
            break;  // uniform: every thread read the same pivot
          }
          const double ljj = sqrt(dj), inv = 1.0 / ljj;
          __syncthreads();
          if (threadIdx.x == 0) blk[j][j] = X::from_real(ljj);
          for (int i = j + 1 + threadIdx.x; i < nb; i += kT) blk[i][j] = X::scale(inv, blk[i][j]);
          __syncthreads();
          const int rest = nb - j - 1;
          for (int t = threadIdx.x; t < rest * rest; t += kT) {
            const int i = j + 1 + t % rest, q = j + 1 + t / rest;
            if (q <= i) blk[i][q] = X::sub(blk[i][q], X::mul(blk[i][j], X::conj(blk[q][j])));
          }
          __syncthreads();
        }
        __syncthreads();
        for (int t = threadIdx.x; t < nb * nb; t += kT) {
          const int i = t % nb, j = t / nb;
          b.L[(p0 + i) + (size_t)(p0 + j) * cap] = j <= i ? blk[i][j] : X::zero();
        }
        if (threadIdx.x == 0 && s_fail) atomicOr(b.werr, kWErrPivot);
      }
      if (!grid_sync(bar, b.werr)) return;
      if (*(volatile int*)b.werr & kWErrPivot) break;  // uniform after the barrier
      // rows below the panel: L[i, p0:p0+nb] = A[i, p0:p0+nb] L_pp^-H
      for (int i = p0 + nb + gtid; i < m1; i += gthreads) {
        D r[kPanel];
#pragma unroll
        for (int q = 0; q < kPanel; ++q) r[q] = q < nb ? ldcg(b.L + i + (size_t)(p0 + q) * cap) : X::zero();
#pragma unroll
        for (int q = 0; q < kPanel; ++q) {
          if (q < nb) {
            D v = r[q];
            for (int t = 0; t < q; ++t) v = X::sub(v, X::mul(r[t], X::conj(ldcg(b.L + (p0 + q) + (size_t)(p0 + t) * cap))));
            r[q] = X::div(v, X::real(ldcg(b.L + (p0 + q) + (size_t)(p0 + q) * cap)));
          }
        }
#pragma unroll
        for (int q = 0; q < kPanel; ++q)
          if (q < nb) b.L[i + (size_t)(p0 + q) * cap] = r[q];
      }
      if (!grid_sync(bar, b.werr)) return;
      // trailing lower triangle
      const int s0 = p0 + nb, R = m1 - s0;
      for (int t = gtid; t < R * R; t += gthreads) {
        const int i = s0 + t % R, j = s0 + t / R;
        if (j > i) continue;
        D acc = ldcg(b.L + i + (size_t)j * cap);
        for (int q = 0; q < nb; ++q)
          acc = X::sub(acc, X::mul(ldcg(b.L + i + (size_t)(p0 + q) * cap), X::conj(ldcg(b.L + j + (size_t)(p0 + q) * cap))));
        b.L[i + (size_t)j * cap] = acc;
      }
      if (!grid_sync(bar, b.werr)) return;
    }
  }
}

// ------------------------------------------------------------------ eigensolver
// Finite check, symmetrised rounding of A, Z = 0.
template <class D>
__global__ void k_w_prep(const Bufs<D>* __restrict__ bufs, const Ctl* __restrict__ ctl, int cap) {
  using X = Cx<D>;
  const int k = blockIdx.y;
  const Ctl c = ctl[k];
  const Bufs<D> b = bufs[k];
  if (c.status != 0 || c.we_m == 0 || *(volatile int*)b.werr != 0) return;
  const int m = c.we_m;
  int bad = 0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < m * m; t += gridDim.x * blockDim.x) {
    const int i = t % m, j = t / m;
    bad |= !X::finite(b.A[i + (size_t)j * cap]);
    if (i == j) {
      b.A[i + (size_t)i * cap] = X::from_real(X::real(b.A[i + (size_t)i * cap]));
    } else if (i > j) {
      const D avg = X::scale(0.5, X::add(b.A[i + (size_t)j * cap], X::conj(b.A[j + (size_t)i * cap])));
      b.A[i + (size_t)j * cap] = avg;
      b.A[j + (size_t)i * cap] = X::conj(avg);
    }
    b.Z[i + (size_t)j * cap] = 0.0;
  }
  if (bad) atomicOr(b.werr, kWErrNonfinite);
}

// Householder reduction of the m x m Hermitian A to tridiagonal form, A = Q T Q^H with
// Q = H_0 H_1 ... H_{m-3}, H_t = I - beta_t v_t v_t^H (v_t in column t of Q below the
// diagonal, beta_t in hv[t]).  One grid barrier per reflector.  Block b owns the columns
// j = b (mod blocks) of A and keeps them in shared memory (slot j / blocks), so the
// matrix-vector products and rank-2 updates of the trailing matrix never leave the SM;
// warp w of a block works on its slots w, w + 8, ...  Step t (L = m - t - 1 rows):
//   every block holds v_t (column t after update t - 1, formed locally);
//   owners form p_j = beta sum_r conj(B[r][j]) v_r for their columns j > t and write p
//   and their partial sums of Re(v^H p) (double-buffered by barrier parity) -- barrier --;
//   every block forms K = beta/2 Re(v^H p) and q = p - K v; owners update their columns
//   j > t + 1, and the owner of column t + 2 writes it to A for every block to read at the
//   next step; column t + 1 (not updated by its owner in this step) is read from A and
//   updated by every block into its next v.  Block 0 records d, the couplings and the
//   reflectors.  At the end the owners write their columns back to A.  Cooperative.
template <class D>
__global__ void __launch_bounds__(kT, 1) k_w_house(const Bufs<D>* __restrict__ bufs, const Ctl* __restrict__ ctl,
                                                   int nk, int cap, int slots, unsigned* bar, double* part) {
  using X = Cx<D>;
  extern __shared__ __align__(16) unsigned char w_sm[];
  D* v = reinterpret_cast<D*>(w_sm);   // reflector of the current step
  D* q = v + cap;
  D* nx = q + cap;                      // column t + 1 being updated into the next v
  D* own = nx + cap;                    // owned columns: slot s at own + s cap
  __shared__ double red[kT / 32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = kT / 32;
  const int G = gridDim.x;
  int parity = 0;   // buffer of p and of the partial sums; alternates at every barrier, across k points
  for (int kk = 0; kk < nk; ++kk) {
    const Ctl c = ctl[kk];
    const Bufs<D> b = bufs[kk];
    if (c.status != 0 || c.we_m == 0 || *(volatile int*)b.werr != 0) continue;   // uniform: set before this launch
    const int m = c.we_m;
    D* A = b.A;
    if (m < 3) continue;
    // owned columns into shared memory; v_0 from column 0 (rows 1..m-1); d_0
    for (int s = 0; s < slots; ++s) {
      const int j = blockIdx.x + G * s;
      if (j >= m) break;
      for (int r = threadIdx.x; r < m; r += kT) own[(size_t)s * cap + r] = ldcg(A + r + (size_t)j * cap);
    }
    for (int i = threadIdx.x; i < m - 1; i += kT) v[i] = ldcg(A + 1 + i);
    if (blockIdx.x == 0 && threadIdx.x == 0) b.td[0] = X::real(ldcg(A));
    __syncthreads();
    for (int t = 0; t + 2 < m; ++t) {
      const int L = m - t - 1;
      double part2 = 0.0;
      for (int i = threadIdx.x; i < L; i += kT) part2 += X::abs2(v[i]);
      part2 = warp_sum_r(part2);
      if (lane == 0) red[warp] = part2;
      __syncthreads();
      double xn2 = 0.0;
      for (int i = 0; i < nw; ++i) xn2 += red[i];
      const double xn = sqrt(xn2);
      const D x0 = v[0];
      __syncthreads();  // red and v[0] read by every thread
      const D* ct1 = A + (t + 1) + (size_t)(t + 1) * cap;   // column t + 1, rows t + 1 ..
      const int o2 = t + 2 < m ? (t + 2) % G : -1;            // owner block of column t + 2
      if (xn == 0.0) {  // nothing to reflect (every block saw the same v): no update
        if ((int)blockIdx.x == o2) {
          const D* src = own + (size_t)((t + 2) / G) * cap;
          for (int r = threadIdx.x; r < L - 1; r += kT) A[(t + 2 + r) + (size_t)(t + 2) * cap] = src[t + 2 + r];
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
          b.hv[t] = X::zero();   // identity reflector
          b.off[t] = X::zero();
          b.td[t + 1] = X::real(ldcg(ct1));
          if (t + 3 == m) b.off[t + 1] = ldcg(ct1 + 1);   // the last coupling
        }
        for (int i = threadIdx.x; i + 1 < L; i += kT) v[i] = ldcg(ct1 + 1 + i);
        if (!grid_sync(bar, b.werr)) return;   // column t + 2 written before it is read
        continue;
      }
      const double ax0 = X::abs(x0);
      const D phase = ax0 > 0.0 ? X::div(x0, ax0) : X::one();
      const D alpha = X::scale(-xn, phase);
      const double beta = 1.0 / (xn * (xn + ax0));
      if (threadIdx.x == 0) v[0] = X::sub(x0, alpha);
      __syncthreads();
      D* pbuf = parity ? b.hq : b.hp;
      double* pp = part + parity * G;
      double pv = 0.0;
      for (int s = warp; s < slots; s += nw) {
        const int j = blockIdx.x + G * s;
        if (j >= m || j <= t) continue;
        const int i = j - t - 1;
        const D* cj = own + (size_t)s * cap + (t + 1);
        D acc = X::zero();
        for (int r = lane; r < L; r += 32) acc = X::add(acc, X::mul(X::conj(cj[r]), v[r]));
        acc = warp_sum_d(acc);
        const D pi = X::scale(beta, acc);
        if (lane == 0) {
          pbuf[i] = pi;
          pv += X::dot_re(v[i], pi);
        }
      }
      pv = warp_sum_r(pv);
      if (lane == 0) red[warp] = pv;
      __syncthreads();
      if (threadIdx.x == 0) {
        double sum = 0.0;
        for (int i = 0; i < nw; ++i) sum += red[i];
        pp[blockIdx.x] = sum;
      }
      if (!grid_sync(bar, b.werr)) return;
      // Re(v^H p) from the blocks' partial sums: loaded once per block, then the same fixed
      // tree in every block (identical K everywhere)
      double pr = 0.0;
      for (int i = threadIdx.x; i < G; i += kT) pr += ldcg(pp + i);
      pr = warp_sum_r(pr);
      if (lane == 0) red[warp] = pr;
      __syncthreads();
      double vp = 0.0;
      for (int i = 0; i < nw; ++i) vp += red[i];
      const double K = 0.5 * beta * vp;
      for (int i = threadIdx.x; i < L; i += kT) q[i] = X::sub(ldcg(pbuf + i), X::scale(K, v[i]));
      __syncthreads();
      // owned columns j > t + 1: B[:, i] -= v conj(q_i) + q conj(v_i); column t + 2 to A
      for (int s = warp; s < slots; s += nw) {
        const int j = blockIdx.x + G * s;
        if (j >= m || j <= t + 1) continue;
        const int i = j - t - 1;
        D* cj = own + (size_t)s * cap + (t + 1);
        const D cq = X::conj(q[i]), cv = X::conj(v[i]);
        for (int r = lane; r < L; r += 32) cj[r] = X::sub(cj[r], X::add(X::mul(v[r], cq), X::mul(q[r], cv)));
        if (j == t + 2) {
          __syncwarp();
          for (int r = lane + 1; r < L; r += 32) A[(t + 1 + r) + (size_t)j * cap] = cj[r];
        }
      }
      // reflector t (v and beta) kept for the back-transformation: v in column t of Q
      if (blockIdx.x == 0) {
        for (int r = threadIdx.x; r < L; r += kT) b.Q[(t + 1 + r) + (size_t)t * cap] = v[r];
        if (threadIdx.x == 0) b.hv[t] = X::from_real(beta);
      }
      // column t + 1 after this update, by every block: its diagonal entry and the next v
      {
        const D cq = X::conj(q[0]), cv = X::conj(v[0]);
        for (int r = threadIdx.x; r < L; r += kT)
          nx[r] = X::sub(ldcg(ct1 + r), X::add(X::mul(v[r], cq), X::mul(q[r], cv)));
      }
      __syncthreads();
      if (blockIdx.x == 0 && threadIdx.x == 0) {
        b.off[t] = alpha;
        b.td[t + 1] = X::real(nx[0]);
        if (t + 3 == m) b.off[t + 1] = nx[1];   // the last coupling is not reflected
      }
      for (int i = threadIdx.x; i + 1 < L; i += kT) v[i] = nx[1 + i];
      __syncthreads();
      parity ^= 1;
    }
    // owned columns back to A (the last diagonal entry is read from there)
    for (int s = 0; s < slots; ++s) {
      const int j = blockIdx.x + G * s;
      if (j >= m) break;
      for (int r = threadIdx.x; r < m; r += kT) A[r + (size_t)j * cap] = own[(size_t)s * cap + r];
    }
    if (!grid_sync(bar, b.werr)) return;   // before the next k point reuses the buffers
  }
}

// Columns per block of the Householder kernel and its shared memory (three vectors and
// the owned columns).
inline int house_slots(int cap, int blocks) { return (cap + blocks - 1) / blocks; }
inline size_t house_smem(int cap, int blocks, size_t dsize) {
  return ((size_t)house_slots(cap, blocks) + 3) * cap * dsize;
}

// Tridiagonal data: d, |e|, phases s (so that T = diag(s)^H T_c diag(s) is real), splits
// where a coupling is negligible, squared couplings, the pivmin safeguard.  One block per k.
template <class D>
__global__ void k_w_tri_setup(const Bufs<D>* __restrict__ bufs, const Ctl* __restrict__ ctl, int cap) {
  using X = Cx<D>;
  const int k = blockIdx.y;
  const Ctl c = ctl[k];
  const Bufs<D> b = bufs[k];
  if (c.status != 0 || c.we_m == 0 || *(volatile int*)b.werr != 0) return;
  const int m = c.we_m;
  // k_w_house left d[0 .. m-2] and every coupling for m >= 3 (the last diagonal entry is in
  // A); smaller problems are tridiagonal already
  if (m < 3) {
    for (int i = threadIdx.x; i < m; i += blockDim.x) b.td[i] = X::real(b.A[i + (size_t)i * cap]);
  } else if (threadIdx.x == 0) {
    b.td[m - 1] = X::real(b.A[(m - 1) + (size_t)(m - 1) * cap]);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (m == 2) b.off[0] = b.A[1];
    D s = X::one();
    b.ph[0] = s;
    for (int i = 0; i + 1 < m; ++i) {
      const double a = X::abs(b.off[i]);
      b.te[i] = a;
      s = a > 0.0 ? X::mul(s, X::div(b.off[i], a)) : s;
      b.ph[i + 1] = s;
    }
    b.te[m - 1] = 0.0;
    int nb = 0;
    b.starts[nb++] = 0;
    double e2max = 1.0;
    for (int i = 0; i + 1 < m; ++i) {
      if (fabs(b.te[i]) <= tri::kUlp * (fabs(b.td[i]) + fabs(b.td[i + 1]))) {
        b.e2[i] = 0.0;
        b.starts[nb++] = i + 1;
      } else {
        b.e2[i] = b.te[i] * b.te[i];
        e2max = fmax(e2max, b.e2[i]);
      }
    }
    b.starts[nb] = m;
    b.wimeta[0] = nb;
    b.wmeta[0] = tri::kSafeMin * e2max;  // pivmin
  }
}

// Eigenvalues by Sturm bisection: one warp per eigenvalue, two shifts per lane per round.
template <class D>
__global__ void __launch_bounds__(kT) k_w_tri_values(const Bufs<D>* __restrict__ bufs, const Ctl* __restrict__ ctl) {
  const int k = blockIdx.y;
  const Ctl c = ctl[k];
  const Bufs<D> b = bufs[k];
  if (c.status != 0 || c.we_m == 0 || *(volatile int*)b.werr != 0) return;
  const int m = c.we_m;
  const int j = blockIdx.x * (kT / 32) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (j >= m) return;
  const int nb = b.wimeta[0];
  const double pivmin = b.wmeta[0];
  const double* d = b.td;
  const double* e = b.te;
  const int bi = tri::block_of(b.starts, nb, j);
  const int s = b.starts[bi], n = b.starts[bi + 1] - s, i = j - s;
  double lo, hi, nrm;
  tri::gershgorin(d, e, s, n, pivmin, &lo, &hi, &nrm);
  constexpr int kShifts = 2, K = 2 * 32;
  const double atol = tri::kUlp * nrm + 2.0 * pivmin;
  for (int it = 0; it < tri::kMaxRounds; ++it) {
    if (hi - lo <= 2.0 * tri::kUlp * fmax(fabs(lo), fabs(hi)) + atol) break;  // uniform in the warp
    const double h = (hi - lo) / (K + 1);
    const int r0 = kShifts * lane;
    double xs[kShifts];
    int cs[kShifts];
#pragma unroll
    for (int q = 0; q < kShifts; ++q) xs[q] = lo + (r0 + q + 1) * h;
    tri::sturm<kShifts>(d, b.e2, s, n, xs, cs);
    int rf = K;
#pragma unroll
    for (int q = kShifts - 1; q >= 0; --q)
      if (cs[q] > i) rf = r0 + q;
    for (int o = 16; o > 0; o >>= 1) rf = min(rf, __shfl_xor_sync(0xffffffffu, rf, o));
    const double nlo = rf > 0 ? lo + rf * h : lo;
    const double nhi = rf < K ? lo + (rf + 1) * h : hi;
    lo = nlo;
    hi = nhi;
  }
  if (lane == 0) b.wu[j] = 0.5 * (lo + hi);
}

// Clusters (consecutive eigenvalues of one block closer than kWideOrtol |T_b|_1), the
// ascending order of all eigenvalues and w in that order.  One block per k.
template <class D>
__global__ void k_w_tri_clusters(const Bufs<D>* __restrict__ bufs, const Ctl* __restrict__ ctl) {
  const int k = blockIdx.y;
  const Ctl c = ctl[k];
  const Bufs<D> b = bufs[k];
  if (c.status != 0 || c.we_m == 0 || *(volatile int*)b.werr != 0) return;
  const int m = c.we_m;
  const int nb = b.wimeta[0];
  const double pivmin = b.wmeta[0];
  if (threadIdx.x == 0) {
    int nc = 0;
    for (int bi = 0; bi < nb; ++bi) {
      const int s = b.starts[bi], n = b.starts[bi + 1] - s;
      double gl, gu, nrm;
      tri::gershgorin(b.td, b.te, s, n, pivmin, &gl, &gu, &nrm);
      const double ortol = kWideOrtol * nrm;
      b.clusters[nc++] = s;
      for (int j = s + 1; j < s + n; ++j)
        if (b.wu[j] - b.wu[j - 1] > ortol) b.clusters[nc++] = j;
    }
    b.clusters[nc] = m;
    b.wimeta[1] = nc;
  }
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    int rank = 0;
    const double di = b.wu[i];
    for (int j = 0; j < m; ++j) rank += (b.wu[j] < di) || (b.wu[j] == di && j < i);
    b.order[rank] = i;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < m; i += blockDim.x) b.w[i] = b.wu[b.order[i]];
}

// Inverse iteration, one thread per eigenvector (tri::eig step 4 with the LU strips in
// global memory, strip entry r of thread j at lu[r cap + j]).  Z[r cap + j].
template <class D>
__global__ void __launch_bounds__(64) k_w_tri_vectors(const Bufs<D>* __restrict__ bufs, const Ctl* __restrict__ ctl,
                                                      int cap) {
  const int k = blockIdx.y;
  const Ctl c = ctl[k];
  const Bufs<D> b = bufs[k];
  if (c.status != 0 || c.we_m == 0 || *(volatile int*)b.werr != 0) return;
  const int m = c.we_m;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  const int nb = b.wimeta[0];
  const double pivmin = b.wmeta[0];
  const double* d = b.td;
  const double* e = b.te;
  const double* wu = b.wu;
  double* Z = b.Z;
  const int ldz = cap;
  const int bi = tri::block_of(b.starts, nb, j);
  const int s = b.starts[bi], n = b.starts[bi + 1] - s;
  if (n == 1) {
    Z[(size_t)s * ldz + j] = 1.0;
    return;
  }
  double gl, gu, onenrm;
  tri::gershgorin(d, e, s, n, pivmin, &gl, &gu, &onenrm);
  const double pertol = 10.0 * tri::kUlp * onenrm, tiny = tri::kUlp * onenrm;
  const double dtpcrt = sqrt(0.1 / n);
  const size_t ps = (size_t)cap;
  double* ur = b.lu + j;
  double* u1 = ur + (size_t)cap * cap;
  double* u2 = u1 + (size_t)cap * cap;
  double* lm = u2 + (size_t)cap * cap;
  int jr = j;
  while (jr > s && wu[jr] - wu[jr - 1] < pertol) --jr;
  const double x = wu[j] + (j - jr) * pertol;
  double ai = d[s] - x, bi_ = e[s], ulast = 0.0;
  bool last_swap = false;
  for (int r = 0; r + 1 < n; ++r) {
    const double ci = e[s + r], an = d[s + r + 1] - x, bn = r + 2 < n ? e[s + r + 1] : 0.0;
    double l, piv;
    if (fabs(ai) >= fabs(ci)) {
      l = ai != 0.0 ? ci / ai : 0.0;
      piv = ai;
      u1[r * ps] = bi_;
      u2[r * ps] = 0.0;
      ai = an - l * bi_;
      bi_ = bn;
    } else {
      l = ai / ci;
      piv = ci;
      u1[r * ps] = an;
      u2[r * ps] = bn;
      ai = bi_ - l * an;
      bi_ = -l * bn;
      if (r + 2 == n) last_swap = true;
    }
    if (fabs(piv) < tiny) piv = piv < 0.0 ? -tiny : tiny;
    ur[r * ps] = 1.0 / piv;
    lm[r * ps] = l;
  }
  if (fabs(ai) < tiny) ai = ai < 0.0 ? -tiny : tiny;
  ulast = fabs(ai);
  ur[(size_t)(n - 1) * ps] = 1.0 / ai;
  double* zc = Z + (size_t)s * ldz + j;
  auto z = [&](int r) -> double& { return zc[(size_t)r * ldz]; };
  double asum = 0.0;
  for (int r = 0; r < n; ++r) {
    const double v = tri::start_entry(j, r);
    z(r) = v;
    asum += fabs(v);
  }
  int checks = 0;
  for (int its = 0; its < tri::kInverseIterations; ++its) {
    const double scl = n * onenrm * fmax(tri::kUlp, ulast) / asum;
    double zr = z(0) * scl;
    for (int r = 0; r + 1 < n; ++r) {
      double zn = z(r + 1) * scl;
      const bool sw = r + 2 < n ? u2[r * ps] != 0.0 : last_swap;
      if (sw) {
        const double t = zr;
        zr = zn;
        zn = t;
      }
      z(r) = zr;
      zr = zn - lm[r * ps] * zr;
    }
    double z1 = zr * ur[(size_t)(n - 1) * ps];
    z(n - 1) = z1;
    double z0 = (z(n - 2) - u1[(size_t)(n - 2) * ps] * z1) * ur[(size_t)(n - 2) * ps];
    z(n - 2) = z0;
    double zmax = fmax(fabs(z1), fabs(z0));
    asum = fabs(z1) + fabs(z0);
    for (int r = n - 3; r >= 0; --r) {
      const double v = (z(r) - u1[r * ps] * z0 - u2[r * ps] * z1) * ur[r * ps];
      z(r) = v;
      z1 = z0;
      z0 = v;
      zmax = fmax(zmax, fabs(v));
      asum += fabs(v);
    }
    if (zmax >= dtpcrt && ++checks > tri::kExtraIterations) break;
  }
  double nn = 0.0;
  for (int r = 0; r < n; ++r) nn += z(r) * z(r);
  const double inv = 1.0 / sqrt(nn);
  for (int r = 0; r < n; ++r) z(r) *= inv;
}

// Each cluster's vectors orthonormalised in order (Gram-Schmidt twice) and every vector's
// largest entry made positive: one warp per cluster.
template <class D>
__global__ void __launch_bounds__(kT) k_w_tri_gs(const Bufs<D>* __restrict__ bufs, const Ctl* __restrict__ ctl, int cap) {
  const int k = blockIdx.y;
  const Ctl c = ctl[k];
  const Bufs<D> b = bufs[k];
  if (c.status != 0 || c.we_m == 0 || *(volatile int*)b.werr != 0) return;
  const int cidx = blockIdx.x * (kT / 32) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  const int nc = b.wimeta[1], nb = b.wimeta[0];
  if (cidx >= nc) return;
  const int ldz = cap;
  const int ja = b.clusters[cidx], jb = b.clusters[cidx + 1];
  const int bi = tri::block_of(b.starts, nb, ja);
  const int s = b.starts[bi], n = b.starts[bi + 1] - s;
  const double* zb = b.Z + (size_t)s * ldz;
  for (int j = ja; j < jb; ++j) {
    double* zc = b.Z + (size_t)s * ldz + j;
    for (int pass = 0; pass < 2 && j > ja; ++pass) {
      for (int qv = ja; qv < j; ++qv) {
        double dot = 0.0;
        for (int r = lane; r < n; r += 32) dot = fma(zc[(size_t)r * ldz], zb[(size_t)r * ldz + qv], dot);
        dot = warp_sum_r(dot);
        for (int r = lane; r < n; r += 32) zc[(size_t)r * ldz] = fma(-dot, zb[(size_t)r * ldz + qv], zc[(size_t)r * ldz]);
        __syncwarp();
      }
      double nn = 0.0;
      for (int r = lane; r < n; r += 32) nn = fma(zc[(size_t)r * ldz], zc[(size_t)r * ldz], nn);
      nn = warp_sum_r(nn);
      const double inv = 1.0 / sqrt(nn);
      for (int r = lane; r < n; r += 32) zc[(size_t)r * ldz] *= inv;
      __syncwarp();
    }
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

// Y[:, c] = H_0 H_1 ... H_{m-3} (s . Z[:, order[c]]) for c < m: kBackCols columns per
// block, one warp per column; each reflector is staged once per block in shared memory
// (double-buffered, one barrier per reflector) and applied by every warp to its column.
constexpr int kBackCols = 6;  // (6 + 2) x 1536 x 16 bytes of shared memory at the largest capacity
template <class D>
__global__ void __launch_bounds__(kT) k_w_back(const Bufs<D>* __restrict__ bufs, const Ctl* __restrict__ ctl, int cap) {
  using X = Cx<D>;
  const int k = blockIdx.y;
  const Ctl c = ctl[k];
  const Bufs<D> b = bufs[k];
  if (c.status != 0 || c.we_m == 0 || *(volatile int*)b.werr != 0) return;
  const int m = c.we_m;
  const int c0 = blockIdx.x * kBackCols;
  if (c0 >= m) return;
  extern __shared__ __align__(16) unsigned char w_sm[];
  D* z = reinterpret_cast<D*>(w_sm);          // [kBackCols][cap]
  D* vb = z + (size_t)kBackCols * cap;        // two reflector buffers of cap
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int col = c0 + warp;
  const bool act = warp < kBackCols && col < m;
  D* zc = z + (size_t)warp * cap;
  if (act) {
    const int src = b.order[col];
    for (int r = lane; r < m; r += 32) zc[r] = X::scale(b.Z[(size_t)r * cap + src], b.ph[r]);
  }
  const int last = m - 3;
  if (last >= 0)
    for (int r = threadIdx.x; r < m - last - 1; r += kT) vb[r] = b.Q[(last + 1 + r) + (size_t)last * cap];
  __syncthreads();
  for (int t = last, buf = 0; t >= 0; --t, buf ^= 1) {
    const int L = m - t - 1;
    const D* v = vb + (size_t)buf * cap;
    // stage the next reflector into the other buffer while this one is applied
    if (t > 0)
      for (int r = threadIdx.x; r < L + 1; r += kT) vb[(size_t)(buf ^ 1) * cap + r] = b.Q[(t + r) + (size_t)(t - 1) * cap];
    const double beta = X::real(b.hv[t]);
    if (act && beta != 0.0) {
      D acc = X::zero();
      for (int r = lane; r < L; r += 32) acc = X::add(acc, X::mul(X::conj(v[r]), zc[t + 1 + r]));
      acc = X::scale(beta, warp_sum_d(acc));
      for (int r = lane; r < L; r += 32) zc[t + 1 + r] = X::sub(zc[t + 1 + r], X::mul(v[r], acc));
    }
    __syncthreads();
  }
  if (act)
    for (int r = lane; r < m; r += 32) b.Y[r + (size_t)col * cap] = zc[r];
}

inline size_t back_smem(int cap, size_t dsize) { return ((size_t)kBackCols + 2) * cap * dsize; }

// LT = L^H (m x m).
template <class D>
__global__ void k_w_adjoint(const Bufs<D>* __restrict__ bufs, const Ctl* __restrict__ ctl, int cap) {
  const int k = blockIdx.y;
  const Ctl c = ctl[k];
  const Bufs<D> b = bufs[k];
  if (c.status != 0 || c.we_m == 0 || *(volatile int*)b.werr != 0) return;
  const int m = c.we_m;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < m * m; t += gridDim.x * blockDim.x) {
    const int i = t % m, j = t / m;
    b.LT[i + (size_t)j * cap] = Cx<D>::conj(b.L[j + (size_t)i * cap]);
  }
}

// ------------------------------------------------------------------ host side
// Shared-memory limits of the kernels above 48 KB and the cooperative grid (one block per
// SM, every one resident).
template <class D>
int prepare(int cap, int* coop_blocks, std::string* err) {
  const int tsm = (int)trsm_smem(cap, sizeof(D));
  int dev0 = 0, sms0 = 0;
  cudaError_t e = cudaGetDevice(&dev0);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms0, cudaDevAttrMultiProcessorCount, dev0);
  if (e == cudaSuccess && house_smem(cap, std::max(sms0, 1), sizeof(D)) > 220 * 1024) {
    *err = "the many-block reduced problem keeps its columns in shared memory: capacity too large for this GPU";
    return BG_EINVAL;
  }
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void*)k_w_house<D>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)house_smem(cap, std::max(sms0, 1), sizeof(D)));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void*)k_w_back<D>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)back_smem(cap, sizeof(D)));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void*)k_w_trsm<D, kSolveBorder>, cudaFuncAttributeMaxDynamicSharedMemorySize, tsm);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void*)k_w_trsm<D, kSolveLeft>, cudaFuncAttributeMaxDynamicSharedMemorySize, tsm);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void*)k_w_trsm<D, kSolveRight>, cudaFuncAttributeMaxDynamicSharedMemorySize, tsm);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void*)k_w_trsm<D, kSolveBack>, cudaFuncAttributeMaxDynamicSharedMemorySize, tsm);
  int dev = 0, sms = 0, occ_h = 0, occ_c = 0;
  if (e == cudaSuccess) e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_h, k_w_house<D>, kT, house_smem(cap, sms, sizeof(D)));
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_c, k_w_chol<D>, kT, 0);
  if (e != cudaSuccess) {
    *err = std::string("many-block reduced problem: ") + cudaGetErrorString(e);
    return BG_EDEVICE;
  }
  if (occ_h < 1 || occ_c < 1 || sms < 1) {
    *err = "the many-block reduced problem cannot place its blocks";
    return BG_EDEVICE;
  }
  *coop_blocks = sms;
  return BG_OK;
}

template <class... A>
void coop_launch(void (*f)(A...), int blocks, size_t smem, cudaStream_t s, A... args) {
  void* argv[] = {&args...};
  cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(f), dim3((unsigned)blocks), dim3(kT), argv, smem, s);
}

// Extension of the factor for every k point with a request (3 launches).
template <class D>
int64_t launch_chol(Bufs<D>* bufs, Ctl* ctl, int nk, int cap, int coop_blocks, unsigned* bar, cudaStream_t s) {
  const dim3 gs((unsigned)((cap + kSolveCols - 1) / kSolveCols), (unsigned)nk);
  k_w_trsm<D, kSolveBorder><<<gs, kT, trsm_smem(cap, sizeof(D)), s>>>(bufs, ctl, cap);
  const unsigned tiles = (unsigned)((cap + kTile - 1) / kTile);
  k_w_border<D><<<dim3(tiles * tiles, (unsigned)nk), kTile * kTile, 0, s>>>(bufs, ctl, cap);
  coop_launch(k_w_chol<D>, coop_blocks, 0, s, (const Bufs<D>*)bufs, (const Ctl*)ctl, nk, cap, bar);
  return 3;
}

// Reduced eigenproblem for every k point with a request (12 launches).
template <class D>
int64_t launch_eig(Bufs<D>* bufs, Ctl* ctl, int nk, int cap, int coop_blocks, unsigned* bar, double* part,
                   cudaStream_t s) {
  const size_t tsm = trsm_smem(cap, sizeof(D));
  const dim3 gs((unsigned)((cap + kSolveCols - 1) / kSolveCols), (unsigned)nk);
  const dim3 gw((unsigned)((cap + 7) / 8), (unsigned)nk);
  k_w_trsm<D, kSolveLeft><<<gs, kT, tsm, s>>>(bufs, ctl, cap);
  k_w_trsm<D, kSolveRight><<<gs, kT, tsm, s>>>(bufs, ctl, cap);
  k_w_prep<D><<<dim3(256, (unsigned)nk), 256, 0, s>>>(bufs, ctl, cap);
  coop_launch(k_w_house<D>, coop_blocks, house_smem(cap, coop_blocks, sizeof(D)), s, (const Bufs<D>*)bufs,
              (const Ctl*)ctl, nk, cap, house_slots(cap, coop_blocks), bar, part);
  k_w_tri_setup<D><<<dim3(1, (unsigned)nk), 256, 0, s>>>(bufs, ctl, cap);
  k_w_tri_values<D><<<gw, kT, 0, s>>>(bufs, ctl);
  k_w_tri_clusters<D><<<dim3(1, (unsigned)nk), 256, 0, s>>>(bufs, ctl);
  k_w_tri_vectors<D><<<dim3((unsigned)((cap + 63) / 64), (unsigned)nk), 64, 0, s>>>(bufs, ctl, cap);
  k_w_tri_gs<D><<<gw, kT, 0, s>>>(bufs, ctl, cap);
  k_w_back<D><<<dim3((unsigned)((cap + kBackCols - 1) / kBackCols), (unsigned)nk), kT, back_smem(cap, sizeof(D)), s>>>(
      bufs, ctl, cap);
  k_w_adjoint<D><<<dim3(256, (unsigned)nk), 256, 0, s>>>(bufs, ctl, cap);
  k_w_trsm<D, kSolveBack><<<gs, kT, tsm, s>>>(bufs, ctl, cap);
  return 12;
}

}  // namespace wide
}  // namespace dv
}  // namespace bg
