// Batched block Davidson over every k point of a k-point set, driven from the device.
//
// The algorithm is the reference Davidson of davidson.cu (crates/dft-solvers/src/
// ref_davidson.rs:117-366 real Gamma ORC rows, ref_davidson_complex.rs:641-1110
// complex), run for all k points of a bg_kset at once:
//   * every large product (rotations V C, Gram blocks V^H W, corrections, the H apply
//     of the correction blocks) is ONE launch over all k points (blockIdx.z = k);
//   * the small reduced problem of each k point -- bordered Cholesky with the pivot
//     rule, A = L^-1 H_r L^-H, Householder tridiagonalisation, the tridiagonal
//     eigenproblem by bisection and inverse iteration, C = L^-H Y -- and every control
//     decision (contraction,
//     dropped corrections, repair, convergence) run in a one-block-per-k "control"
//     kernel, which writes the dimensions and pointers of the next large products into
//     per-k descriptors in device memory;
//   * so one iteration is a fixed sequence of launches whose work depends only on
//     device state: it is captured once as a CUDA graph and replayed until every k
//     point has finished (the host reads one status word per replay).
// Branches that a k point does not take this iteration (contraction, repair) are
// launches whose blocks for that k point return at once.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

#include "blas_dev.cuh"
#include "gemm_tc.cuh"
#include "gemm_tiles.cuh"
#include "tridiag_dev.cuh"
#include "op_internal.h"

namespace bg {
namespace dv {

constexpr double kEps = 2.220446049250313e-16;
constexpr double kPivotRatioMin = kEps / 1e-12;   // crates/dft-solvers/src/lean_davidson.rs:62-70
constexpr double kDependence = 1e-12;             // crates/dft-numerics/src/linalg.rs:12
constexpr int kCtlThreads = 256;
// Precision form: the tensor-core phase of a solve hands over to FP64 once every active
// band's residual |HX_j - lambda_j X_j| is below this.
constexpr double kHandoverResidual = 1e-4;
// Iterations without a new smallest Ritz change after which the learned preconditioner
// gives way to TPA (the host-driven solver's rule).
constexpr int kLearnedStall = 5;
// A tensor-phase iteration after which the occupied bands' largest |r|^2 is not below
// this fraction of the best so far (|r| down by less than 30 %) has stalled.
constexpr double kStallFactor = 0.49;
// The tensor phase's own convergence ends a solve only for thresholds (Ha) at or above
// this; below it the FP64 phase judges convergence.  Chosen by measurement: with solves
// ended this way down to 1e-6 Ha the Si64 and Si216 SCF energies stayed within the SCF
// threshold's own accuracy of the FP64 SCF's.
constexpr double kTensorOnlyThreshold = 1e-6;

// Errors recorded by a k point's control kernel (status = -id).
enum : int {
  kErrStartDependent = 1,
  kErrBasisDependent,
  kErrNonfiniteCorrection,
  kErrCapacity,
  kErrRepairDependent,
  kErrEigen,
  kErrTimeout,
};

// ------------------------------------------------------------------ scalar helpers
template <class D>
struct Cx;
template <>
struct Cx<double> {
  __device__ static double zero() { return 0.0; }
  __device__ static double one() { return 1.0; }
  __device__ static double real(double v) { return v; }
  __device__ static double from_real(double v) { return v; }
  __device__ static double conj(double a) { return a; }
  __device__ static double mul(double a, double b) { return a * b; }
  __device__ static double sub(double a, double b) { return a - b; }
  __device__ static double add(double a, double b) { return a + b; }
  __device__ static double scale(double s, double a) { return s * a; }
  __device__ static double abs2(double a) { return a * a; }
  __device__ static double abs(double a) { return fabs(a); }
  __device__ static double neg(double a) { return -a; }
  __device__ static bool finite(double a) { return isfinite(a); }
  __device__ static double div(double a, double r) { return a / r; }
  __device__ static double dot_re(double a, double b) { return a * b; }
  __device__ static double shfl_down(double a, int o) { return __shfl_down_sync(0xffffffffu, a, o); }
  __device__ static double shfl_xor(double a, int o) { return __shfl_xor_sync(0xffffffffu, a, o); }
};
template <>
struct Cx<double2> {
  __device__ static double2 zero() { return make_double2(0.0, 0.0); }
  __device__ static double2 one() { return make_double2(1.0, 0.0); }
  __device__ static double real(double2 v) { return v.x; }
  __device__ static double2 from_real(double v) { return make_double2(v, 0.0); }
  __device__ static double2 conj(double2 a) { return make_double2(a.x, -a.y); }
  __device__ static double2 mul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
  }
  __device__ static double2 sub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
  __device__ static double2 add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
  __device__ static double2 scale(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
  __device__ static double abs2(double2 a) { return a.x * a.x + a.y * a.y; }
  __device__ static double abs(double2 a) { return hypot(a.x, a.y); }
  __device__ static double2 neg(double2 a) { return make_double2(-a.x, -a.y); }
  __device__ static bool finite(double2 a) { return isfinite(a.x) && isfinite(a.y); }
  __device__ static double2 div(double2 a, double r) { return make_double2(a.x / r, a.y / r); }
  __device__ static double dot_re(double2 a, double2 b) { return a.x * b.x + a.y * b.y; }  // Re(conj(a) b)
  __device__ static double2 shfl_down(double2 a, int o) {
    return make_double2(__shfl_down_sync(0xffffffffu, a.x, o), __shfl_down_sync(0xffffffffu, a.y, o));
  }
  __device__ static double2 shfl_xor(double2 a, int o) {
    return make_double2(__shfl_xor_sync(0xffffffffu, a.x, o), __shfl_xor_sync(0xffffffffu, a.y, o));
  }
};

// ------------------------------------------------------------------ device state
// Per-k buffers (device pointers; an array of these lives in device memory).
template <class D>
struct Bufs {
  D *V, *HV, *X, *HX, *E, *Er;   // rows x cap, ld rows
  D *S, *Hr, *L, *C, *A, *Y, *P; // cap x cap, ld cap
  D *Q;                          // Householder accumulation, cap x cap
  double* Z;                     // tridiagonal eigenvectors, cap x cap (real)
  double *w, *old, *lam, *norms, *scale, *td, *te;  // cap
  double* rnorm;                 // cap: |HX_j - lambda_j X_j|^2 of the active bands
  D* off;                        // cap: Householder off-diagonal
  D* ph;                         // cap: phases of the real tridiagonal
  D *hv, *hp, *hq;               // cap: Householder vectors
  int *active, *map, *conv, *order;  // cap
  D* part;                       // split-K partials
  double *e2, *wu;               // cap: tridiagonal solver (squared couplings, eigenvalues by block)
  int *starts, *clusters;        // cap + 1: its blocks and clusters
  const double* diag;            // rows
  int rows;
  // reduced problem on many blocks (large capacities): L^H, inverse-iteration strips
  // (4 cap x cap doubles), error bits, tridiagonal metadata (pivmin; block and cluster counts)
  D* LT;
  double* lu;
  int* werr;
  double* wmeta;
  int* wimeta;
};

// Per-k control scalars.
struct Ctl {
  int m, nact, kept, status, iterations;
  int contract, repair, need_repair;
  int reduced_solves, h_calls, h_columns, repairs, contractions, dropped;
  // requests to the many-block reduced problem: extend the factor from wc_m0 to wc_m1
  // columns, solve the reduced problem of we_m columns (0: none)
  int wc_m0, wc_m1, we_m;
  // precision form: iterations without a new smallest residual, and that residual (squared)
  int stall;
  double best_res;
  // the preconditioner in use (the learned one gives way to TPA when the solve stalls),
  // the smallest largest-Ritz-change so far and the iterations since it fell
  int precond, pstall, fallbacks;
  double best_change;
};

// Descriptors of the large products of one slot (written by the control kernel).
template <class D>
// prec 1: the product runs as BF16x3 on the tensor cores (precision form), else FP64.
struct NN {  // C[:, 0:n] (+)= A[:, 0:k] B, B k x n (ld ldb); A and C ld rows
  const D* A;
  const D* B;
  D* C;
  int ldb, n, k, accumulate;
  int prec;
};
template <class D>
struct TN {  // G[0:m, 0:n] (ld ldg) = A[:, 0:m]^H B[:, 0:n]
  const D* A;
  const D* B;
  D* G;
  int ldg, m, n;
  int prec;
};
template <class D>
struct CP {  // dst[:, c] = src[:, c] (scale[c] src[:, map[c]] when pick)
  const D* src;
  D* dst;
  int cols, pick;
};

// Options shared by every k point (crates/dft-solvers/src/ref_davidson.rs:39-77).
struct Opts {
  int n, cap, occupied, first_step, max_iterations;
  double threshold;
  int preconditioner;
  int smem_matrices;  // the control kernel keeps A, Y, Q, Z in shared memory
  int fp32;           // H applies with the FP32 local part
  int wide;           // the reduced problem runs on many blocks (wide_rr.cuh)
  int tensor;         // precision form: tensor-core applies, H Grams and rotations
  double handover;    // precision form: stop once every active band's residual is below
  int want_hx;        // the final phase also forms H X = HV C[:, :n]
};

// ------------------------------------------------------------------ block-wide small algebra
// Every routine below is called by all threads of a control block (kCtlThreads) and
// ends with the block synchronised.

__device__ __forceinline__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double t = 0.0;
  for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
  __syncthreads();
  return t;
}

// Block sum with one barrier: warp partials go to `slot` (32 doubles) and every thread adds
// them in warp order.  A slot may be written again only after another barrier, so two
// successive calls use different slots unless a barrier lies between them.
__device__ __forceinline__ double block_sum1(double v, double* slot) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) slot[warp] = v;
  __syncthreads();
  double t = 0.0;
  for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += slot[i];
  return t;
}

template <class D>
__device__ __forceinline__ D warp_sum(D v) {
  for (int o = 16; o > 0; o >>= 1) v = Cx<D>::add(v, Cx<D>::shfl_down(v, o));
  return v;
}

// Extend the lower Cholesky factor L of S (both ld, columns 0..m0-1 of L valid) to
// columns m0..m-1 with the reference's pivot rule (squared pivot over the overlap
// diagonal >= eps / 1e-12, crates/dft-solvers/src/lean_davidson.rs:62-70).  The part of
// the new rows left of m0 is a right-looking forward substitution, parallel over the new
// rows and columns; the new diagonal block is factored right-looking by the whole block.
template <class D>
__device__ bool chol_extend(const D* S, int ld, D* L, int m0, int m, int* flag) {
  using X = Cx<D>;
  if (m0 > 0) {
    // right-looking: L[j][k] holds S[j][k] minus the updates of columns p < k until
    // column k is divided by its pivot; every step is parallel over the new rows
    const int nr = m - m0;
    for (int t = threadIdx.x; t < nr * m0; t += blockDim.x) {
      const int j = m0 + t % nr, k = t / nr;
      L[j + (size_t)k * ld] = S[j + (size_t)k * ld];
    }
    __syncthreads();
    for (int p = 0; p < m0; ++p) {
      const double piv = X::real(L[p + (size_t)p * ld]);
      for (int j = m0 + (int)threadIdx.x; j < m; j += blockDim.x)
        L[j + (size_t)p * ld] = X::div(L[j + (size_t)p * ld], piv);
      __syncthreads();
      const int cols = m0 - p - 1;
      for (int t = threadIdx.x; t < nr * cols; t += blockDim.x) {
        const int j = m0 + t % nr, k = p + 1 + t / nr;
        L[j + (size_t)k * ld] =
            X::sub(L[j + (size_t)k * ld], X::mul(L[j + (size_t)p * ld], X::conj(L[k + (size_t)p * ld])));
      }
      __syncthreads();
    }
  }
  __syncthreads();
  // the new diagonal block: D = S22 - L21 L21^H in the lower triangle of L's block, then a
  // right-looking factorisation, one pivot per step (its ratio to the overlap diagonal
  // checked by the reference's rule), the column below scaled and the trailing lower
  // triangle updated in parallel
  const int nr = m - m0;
  for (int t = threadIdx.x; t < nr * nr; t += blockDim.x) {
    const int j = m0 + t % nr, k = m0 + t / nr;
    if (k > j) {
      L[j + (size_t)k * ld] = X::zero();
      continue;
    }
    D acc = S[j + (size_t)k * ld];
    for (int p = 0; p < m0; ++p) acc = X::sub(acc, X::mul(L[j + (size_t)p * ld], X::conj(L[k + (size_t)p * ld])));
    L[j + (size_t)k * ld] = acc;
  }
  for (int t = threadIdx.x; t < m0 * nr; t += blockDim.x)  // above the new block
    L[t % m0 + (size_t)(m0 + t / m0) * ld] = X::zero();
  if (threadIdx.x == 0) *flag = 1;
  __syncthreads();
  for (int j = m0; j < m; ++j) {
    const double sjj = X::real(S[j + (size_t)j * ld]);
    const double dj = X::real(L[j + (size_t)j * ld]);
    const double ratio = dj / sjj;
    if (!(ratio >= kPivotRatioMin) || !isfinite(ratio)) {
      if (threadIdx.x == 0) *flag = 0;
      break;  // uniform: every thread read the same pivot
    }
    const double ljj = sqrt(dj), inv = 1.0 / ljj;
    __syncthreads();  // every thread has read the pivot before it is replaced
    if (threadIdx.x == 0) L[j + (size_t)j * ld] = X::from_real(ljj);
    for (int i = j + 1 + (int)threadIdx.x; i < m; i += blockDim.x)
      L[i + (size_t)j * ld] = X::scale(inv, L[i + (size_t)j * ld]);
    __syncthreads();
    const int rest = m - j - 1;
    for (int t = threadIdx.x; t < rest * rest; t += blockDim.x) {
      const int i = j + 1 + t % rest, k = j + 1 + t / rest;
      if (k <= i)
        L[i + (size_t)k * ld] = X::sub(L[i + (size_t)k * ld], X::mul(L[i + (size_t)j * ld], X::conj(L[k + (size_t)j * ld])));
    }
    __syncthreads();
  }
  __syncthreads();
  const bool ok = *flag != 0;
  __syncthreads();
  return ok;
}

// Lanes that share one column of a triangular solve, or one row or column of a
// Householder product (partial sums combined by shuffles within the group).
constexpr int kSolveLanes = 4;
constexpr int kHouseLanes = 8;

template <class D, int G>
__device__ __forceinline__ D group_sum(D v) {
  for (int o = G / 2; o > 0; o >>= 1) v = Cx<D>::add(v, Cx<D>::shfl_xor(v, o));
  return v;
}

// rdiag[i] = 1 / L[i][i] (the real diagonal of a Cholesky factor).
template <class D>
__device__ void reciprocal_diagonal(const D* L, int ldl, int m, double* rdiag) {
  for (int i = threadIdx.x; i < m; i += blockDim.x) rdiag[i] = 1.0 / Cx<D>::real(L[i + (size_t)i * ldl]);
  __syncthreads();
}

// B <- L^-1 B (L lower m x m, B m x ncols): kSolveLanes lanes per column split each
// row's dot product; rdiag from reciprocal_diagonal.
template <class D>
__device__ void trsm_lower(const D* L, int ldl, D* B, int ldb, int m, int ncols, const double* rdiag) {
  using X = Cx<D>;
  constexpr int G = kSolveLanes;
  const int g = threadIdx.x % G, per = blockDim.x / G;
  for (int c0 = 0; c0 < ncols; c0 += per) {
    const int c = c0 + threadIdx.x / G;
    const bool act = c < ncols;
    D* b = B + (size_t)(act ? c : 0) * ldb;
    for (int i = 0; i < m; ++i) {
      D part = X::zero();
      if (act)
        for (int k = g; k < i; k += G) part = X::add(part, X::mul(L[i + (size_t)k * ldl], b[k]));
      part = group_sum<D, G>(part);
      if (act && g == 0) b[i] = X::scale(rdiag[i], X::sub(b[i], part));
      __syncwarp();
    }
  }
  __syncthreads();
}

// B <- L^-H B.
template <class D>
__device__ void trsm_lower_adjoint(const D* L, int ldl, D* B, int ldb, int m, int ncols, const double* rdiag) {
  using X = Cx<D>;
  constexpr int G = kSolveLanes;
  const int g = threadIdx.x % G, per = blockDim.x / G;
  for (int c0 = 0; c0 < ncols; c0 += per) {
    const int c = c0 + threadIdx.x / G;
    const bool act = c < ncols;
    D* b = B + (size_t)(act ? c : 0) * ldb;
    for (int i = m - 1; i >= 0; --i) {
      D part = X::zero();
      if (act)
        for (int k = i + 1 + g; k < m; k += G) part = X::add(part, X::mul(X::conj(L[k + (size_t)i * ldl]), b[k]));
      part = group_sum<D, G>(part);
      if (act && g == 0) b[i] = X::scale(rdiag[i], X::sub(b[i], part));
      __syncwarp();
    }
  }
  __syncthreads();
}

// dst (m x m, ld) = conj(src)^T.
template <class D>
__device__ void adjoint(const D* src, D* dst, int ld, int m) {
  for (int t = threadIdx.x; t < m * m; t += blockDim.x) {
    const int i = t % m, j = t / m;
    dst[i + (size_t)j * ld] = Cx<D>::conj(src[j + (size_t)i * ld]);
  }
  __syncthreads();
}

// Hermitian eigensolver of the m x m matrix A (ld lda, overwritten), eigenvalues
// ascending in w, eigenvectors in V (ld ldv): Householder reduction to a Hermitian
// tridiagonal matrix and the unitary diagonal scaling to a real symmetric one as in the
// host solver (dense_host.h heev), whose implicit QL is a serial rotation chase; here
// the tridiagonal eigenpairs come from tri::eig (bisection by lane groups, inverse
// iteration by clusters), then the back-transformation.  Work arrays come from the k
// point's Bufs (ld ldq = cap).  The eigenpairs agree with the host solver's to rounding
// (eigenvectors of a degenerate level up to a rotation inside it, as between any two
// stable eigensolvers).  Returns false on a non-finite input.
template <class D>
__device__ bool heev(D* A, int lda, int m, double* w, D* V, int ldv, const Bufs<D>& b, int ldq, double* red,
                     int* sh) {
  using X = Cx<D>;
  // finite input
  int bad = 0;
  for (int t = threadIdx.x; t < m * m; t += blockDim.x) bad |= !X::finite(A[(t % m) + (size_t)(t / m) * lda]);
  if (block_sum((double)bad, red) != 0.0) return false;
  // symmetrise the rounding of the input
  for (int t = threadIdx.x; t < m * m; t += blockDim.x) {
    const int i = t % m, j = t / m;
    if (i == j) {
      A[i + (size_t)i * lda] = X::from_real(X::real(A[i + (size_t)i * lda]));
    } else if (i > j) {
      const D avg = X::scale(0.5, X::add(A[i + (size_t)j * lda], X::conj(A[j + (size_t)i * lda])));
      A[i + (size_t)j * lda] = avg;
      A[j + (size_t)i * lda] = X::conj(avg);
    }
  }
  D* Q = b.Q;
  for (int t = threadIdx.x; t < m * m; t += blockDim.x) {
    const int i = t % m, j = t / m;
    Q[i + (size_t)j * ldq] = i == j ? X::one() : X::zero();
  }
  for (int t = threadIdx.x; t < m; t += blockDim.x) b.off[t] = X::zero();
  __syncthreads();
  D* v = b.hv;
  D* p = b.hp;
  // Q is stored transposed (Q[c + r ldq] holds row r, column c), so that the reflector
  // update of each row reads contiguous entries.
  const int hg = threadIdx.x % kHouseLanes, hper = blockDim.x / kHouseLanes;
  // Two block reductions per step and no other barrier: p = beta B v reads v straight from
  // the column (v_0 = x_0 - alpha) and sums Re(v^H p) on the way (the K reduction's barrier
  // also publishes p and v); the rank-2 update forms q = p - K v on the fly and sums the
  // next column's squared norm, whose reduction closes the step.  red and red + 32 take
  // the two reductions in turn, so a slot is never rewritten while it is still read.
  double xn2 = 0.0;
  if (m > 2) {
    double part = 0.0;
    for (int i = threadIdx.x; i < m - 1; i += blockDim.x) part += X::abs2(A[1 + i]);
    xn2 = block_sum1(part, red + 32);
  }
  for (int k = 0; k + 2 < m; ++k) {
    const int L = m - k - 1;
    D* x = A + (k + 1) + (size_t)k * lda;
    const double xn = sqrt(xn2);
    if (xn == 0.0) {
      if (threadIdx.x == 0) b.off[k] = X::zero();
      double part = 0.0;
      for (int i = threadIdx.x; i + 1 < L; i += blockDim.x) part += X::abs2(A[(k + 2 + i) + (size_t)(k + 1) * lda]);
      __syncthreads();  // the previous reduction in red + 32 has been read by every thread
      xn2 = block_sum1(part, red + 32);
      continue;
    }
    const D x0 = x[0];
    const double ax0 = X::abs(x0);
    const D phase = ax0 > 0.0 ? X::div(x0, ax0) : X::one();
    const D alpha = X::scale(-xn, phase);
    const D v0 = X::sub(x0, alpha);
    for (int i = threadIdx.x; i < L; i += blockDim.x) v[i] = i == 0 ? v0 : x[i];
    // |v|^2 = |x|^2 - |x0|^2 + (|x0| + |x|)^2
    const double beta = 1.0 / (xn * (xn + ax0));
    // p = beta B v, entry i from column i of the Hermitian B (contiguous)
    double part = 0.0;
    for (int i0 = 0; i0 < L; i0 += hper) {
      const int i = i0 + threadIdx.x / kHouseLanes;
      D acc = X::zero();
      if (i < L) {
        const D* col = A + (k + 1) + (size_t)(k + 1 + i) * lda;
        for (int j = hg; j < L; j += kHouseLanes) acc = X::add(acc, X::mul(X::conj(col[j]), j == 0 ? v0 : x[j]));
      }
      acc = group_sum<D, kHouseLanes>(acc);
      if (i < L && hg == 0) {
        const D pi = X::scale(beta, acc);
        p[i] = pi;
        part += X::dot_re(i == 0 ? v0 : x[i], pi);
      }
    }
    const double K = 0.5 * beta * block_sum1(part, red);
    double nxt = 0.0;
    for (int t = threadIdx.x; t < L * L; t += blockDim.x) {
      const int i = t % L, j = t / L;
      const D qi = X::sub(p[i], X::scale(K, v[i])), qj = X::sub(p[j], X::scale(K, v[j]));
      D& a = A[(k + 1 + i) + (size_t)(k + 1 + j) * lda];
      a = X::sub(a, X::add(X::mul(v[i], X::conj(qj)), X::mul(qi, X::conj(v[j]))));
      if (j == 0 && i >= 1) nxt += X::abs2(a);
    }
    if (threadIdx.x == 0) b.off[k] = alpha;
    for (int i = threadIdx.x; i < L; i += blockDim.x) {
      x[i] = X::zero();
      A[k + (size_t)(k + 1 + i) * lda] = X::zero();
    }
    // Q <- Q H on columns k+1..m-1, one row per lane group
    for (int r0 = 0; r0 < m; r0 += hper) {
      const int r = r0 + threadIdx.x / kHouseLanes;
      D* row = Q + (k + 1) + (size_t)(r < m ? r : 0) * ldq;
      D acc = X::zero();
      if (r < m)
        for (int j = hg; j < L; j += kHouseLanes) acc = X::add(acc, X::mul(row[j], v[j]));
      acc = X::scale(beta, group_sum<D, kHouseLanes>(acc));
      if (r < m)
        for (int j = hg; j < L; j += kHouseLanes) row[j] = X::sub(row[j], X::mul(acc, X::conj(v[j])));
    }
    xn2 = block_sum1(nxt, red + 32);  // the next column's |x|^2; its barrier closes the step
  }
  double* d = b.td;
  double* e = b.te;
  D* s = b.ph;
  if (threadIdx.x == 0) {
    if (m >= 2) b.off[m - 2] = A[(m - 1) + (size_t)(m - 2) * lda];
    for (int i = 0; i < m; ++i) d[i] = X::real(A[i + (size_t)i * lda]);
    s[0] = X::one();
    for (int i = 0; i + 1 < m; ++i) {
      const double a = X::abs(b.off[i]);
      e[i] = a;
      s[i + 1] = a > 0.0 ? X::mul(s[i], X::div(b.off[i], a)) : s[i];
    }
    e[m - 1] = 0.0;
  }
  __syncthreads();
  double* Z = b.Z;
  // A (read into d, e) and V (written by the back-transform below) are free here: they
  // hold the inverse iteration's LU strips
  const int mat_doubles = (int)((size_t)ldq * ldq * sizeof(D) / sizeof(double));
  tri::eig<kCtlThreads>(m, d, e, b.e2, b.wu, b.starts, b.clusters, Z, ldq, reinterpret_cast<double*>(A), mat_doubles,
                        reinterpret_cast<double*>(V), mat_doubles, sh);
  const double* wu = b.wu;
  // stable ascending order of the eigenvalues (rank of each entry)
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    int rank = 0;
    const double di = wu[i];
    for (int j = 0; j < m; ++j) rank += (wu[j] < di) || (wu[j] == di && j < i);
    b.order[rank] = i;
  }
  __syncthreads();
  for (int c = threadIdx.x; c < m; c += blockDim.x) w[c] = wu[b.order[c]];
  // V = Q diag(s) Z[:, order]: lanes take consecutive columns (Z row-major, Q transposed)
  for (int t = threadIdx.x; t < m * m; t += blockDim.x) {
    const int c = t % m, r = t / m;
    const int src = b.order[c];
    D acc = X::zero();
    for (int k = 0; k < m; ++k) acc = X::add(acc, X::mul(Q[k + (size_t)r * ldq], X::scale(Z[(size_t)k * ldq + src], s[k])));
    V[r + (size_t)c * ldv] = acc;
  }
  __syncthreads();
  return true;
}

// Reduced eigenproblem of the first m basis columns: A = L^-1 H_r L^-H, A Y = Y diag(w),
// C = L^-H Y (crates/dft-numerics/src/linalg.rs:234-444 for the complex form,
// crates/dft-solvers/src/ref_davidson/workspace.rs:385-499 for the real one).
template <class D>
__device__ bool eigen(const Bufs<D>& b, int cap, int m, double* red, int* sh) {
  for (int t = threadIdx.x; t < m * m; t += blockDim.x) {
    const int i = t % m, j = t / m;
    b.A[i + (size_t)j * cap] = b.Hr[i + (size_t)j * cap];
  }
  __syncthreads();
  reciprocal_diagonal(b.L, cap, m, b.e2);
  trsm_lower(b.L, cap, b.A, cap, m, m, b.e2);
  adjoint(b.A, b.Y, cap, m);
  trsm_lower(b.L, cap, b.Y, cap, m, m, b.e2);
  adjoint(b.Y, b.A, cap, m);
  if (!heev(b.A, cap, m, b.w, b.Y, cap, b, cap, red, sh)) return false;
  reciprocal_diagonal(b.L, cap, m, b.e2);   // heev used e2 as scratch
  trsm_lower_adjoint(b.L, cap, b.Y, cap, m, m, b.e2);
  for (int t = threadIdx.x; t < m * m; t += blockDim.x) {
    const int i = t % m, j = t / m;
    b.C[i + (size_t)j * cap] = b.Y[i + (size_t)j * cap];
  }
  __syncthreads();
  return true;
}

// ------------------------------------------------------------------ batched large products
// Descriptor arrays are laid out [slot][k]; blockIdx.z enumerates (slot, k).

// C (+)= A B for every (slot, k) with a non-empty descriptor; 64 x 64 tiles.  blockIdx.x
// runs over the column tiles, so the blocks that read one 64-row slice of the tall A
// launch together and share it in L2.
template <class D>
__global__ void __launch_bounds__(256, 2) k_dv_nn(const Bufs<D>* __restrict__ bufs, const NN<D>* __restrict__ desc,
                                                  int nk) {
  const int z = blockIdx.z, k = z % nk;
  const NN<D> d = desc[z];
  const int rows = bufs[k].rows;
  const int64_t r0 = (int64_t)blockIdx.y * 64;
  const int j0 = blockIdx.x * 64;
  if (d.n <= 0 || d.prec || j0 >= d.n || r0 >= rows) return;
  tiles::nn_tile64_mma<D, true>(d.A, rows, d.B, d.ldb, d.C, rows, rows, d.n, d.k, r0, j0, d.accumulate != 0);
}

// Split-K partial Gram products: part[slot][s][j][i] = sum over row slice s of
// conj(A[r][i]) B[r][j]; blockIdx.z = (slot * nk + k) * ks + s.
template <class D>
__global__ void __launch_bounds__(256, 2) k_dv_tn(const Bufs<D>* __restrict__ bufs, const TN<D>* __restrict__ desc, int nk,
                                              int ks, int64_t slot_elems) {
  const int zz = blockIdx.z / ks, sidx = blockIdx.z % ks;
  const int slot = zz / nk, k = zz % nk;
  const TN<D> d = desc[zz];
  if (d.m <= 0 || d.n <= 0 || d.prec || (int)blockIdx.x * 48 >= d.m || (int)blockIdx.y * 48 >= d.n) return;
  const int64_t rows = bufs[k].rows;
  int64_t chunk = (rows + ks - 1) / ks;
  chunk = ((chunk + 31) / 32) * 32;
  const int64_t r0 = min(rows, (int64_t)sidx * chunk), r1 = min(rows, r0 + chunk);
  D* part = bufs[k].part + slot * slot_elems + (int64_t)sidx * d.m * d.n;
  tiles::tn_tile48_mma<D>(d.A, rows, d.B, rows, blockIdx.x * 48, blockIdx.y * 48, d.m, d.n, r0, r1, part, d.m);
}

// G[i + j ldg] = sum_s part[slot][s][j][i] in slice order.
template <class D>
__global__ void k_dv_tn_sum(const Bufs<D>* __restrict__ bufs, const TN<D>* __restrict__ desc, int nk, int ks,
                            int64_t slot_elems) {
  const int zz = blockIdx.z, slot = zz / nk, k = zz % nk;
  const TN<D> d = desc[zz];
  if (d.m <= 0 || d.n <= 0 || d.prec) return;
  const D* part = bufs[k].part + slot * slot_elems;
  const int64_t total = (int64_t)d.m * d.n;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = t / d.m, i = t - j * d.m;
    D acc = Arith<D>::zero();
    for (int q = 0; q < ks; ++q) acc = Arith<D>::add(acc, part[(int64_t)q * total + t]);
    d.G[i + j * d.ldg] = acc;
  }
}

// dst[:, c] = src[:, c], or scale[c] src[:, map[c]] for a pick; blockIdx.y = column.  A
// thread moves kCopyUnroll rows per pass with its loads issued together, so a block's
// descriptor reads are paid for once per kCopyUnroll x 256 rows.
constexpr int kCopyUnroll = 4;
template <class D>
__global__ void k_dv_copy(const Bufs<D>* __restrict__ bufs, const CP<D>* __restrict__ desc, int nk) {
  const int z = blockIdx.z, k = z % nk;
  const CP<D> d = desc[z];
  const int c = blockIdx.y;
  if (c >= d.cols) return;
  const Bufs<D>& b = bufs[k];
  const int64_t rows = b.rows;
  const D* src = d.src + (int64_t)(d.pick ? b.map[c] : c) * rows;
  D* dst = d.dst + (int64_t)c * rows;
  const double sc = d.pick ? b.scale[c] : 1.0;
  const int64_t span = (int64_t)blockDim.x * kCopyUnroll;
  for (int64_t r0 = blockIdx.x * span + threadIdx.x; r0 < rows; r0 += (int64_t)gridDim.x * span) {
    D v[kCopyUnroll];
#pragma unroll
    for (int u = 0; u < kCopyUnroll; ++u) {
      const int64_t r = r0 + (int64_t)u * blockDim.x;
      if (r < rows) v[u] = src[r];
    }
#pragma unroll
    for (int u = 0; u < kCopyUnroll; ++u) {
      const int64_t r = r0 + (int64_t)u * blockDim.x;
      if (r < rows) dst[r] = d.pick ? Arith<D>::scale(sc, v[u]) : v[u];
    }
  }
}

// Dense test operators: y[:, 0:cols] = H x for every k point, cols read from dyn.
template <class D>
__global__ void __launch_bounds__(128) k_dv_dense(const D* const* __restrict__ H, const Bufs<D>* __restrict__ bufs,
                                                  const DynCols* __restrict__ dyn) {
  const int k = blockIdx.z;
  const DynCols dc = dyn[k];
  const int rows = bufs[k].rows;
  const int64_t r0 = (int64_t)blockIdx.x * 64;
  const int j0 = blockIdx.y * 32;
  if (j0 >= dc.cols || r0 >= rows) return;
  tiles::nn_tile<D>(H[k], rows, reinterpret_cast<const D*>(dc.x), rows, reinterpret_cast<D*>(dc.y), rows, rows,
                    dc.cols, rows, r0, j0, false);
}

// Corrections of the active bands of every running k point (correction_column with the
// solver's preconditioner), norms[j] = |Er[:, j]|^2.
template <class D>
__global__ void __launch_bounds__(256) k_dv_corrections(const Bufs<D>* __restrict__ bufs, const Ctl* __restrict__ ctl,
                                                        const Opts* __restrict__ opts,
                                                        const __nv_bfloat16* __restrict__ net) {
  __shared__ double red[256];
  __shared__ float wnet[learned::kParams];
  const int j = blockIdx.x, k = blockIdx.y;
  const Ctl& c = ctl[k];
  if (c.status != 0 || j >= c.nact) return;
  const int kind = c.precond;
  const Bufs<D>& b = bufs[k];
  const int64_t rows = b.rows;
  double r2 = 0.0;
  double n2;
  if (kind == BG_PRECOND_LEARNED) {  // block-uniform: one k point per block row
    learned::load_params(net, wnet);
    n2 = correction_column<D, true>(b.X + j * rows, b.HX + j * rows, b.diag, b.lam[j], kind, rows, b.Er + j * rows,
                                    red, wnet, &r2);
  } else {
    n2 = correction_column(b.X + j * rows, b.HX + j * rows, b.diag, b.lam[j], kind, rows, b.Er + j * rows, red,
                           nullptr, &r2);
  }
  if (threadIdx.x == 0) {
    b.norms[j] = n2;
    b.rnorm[j] = r2;
  }
}

// Tensor-core descriptors of the products marked prec = 1 (complex blocks): one thread per
// (slot, k point); the others get empty descriptors.
template <class D>
__global__ void k_dv_tc_descs(const Bufs<D>* __restrict__ bufs, const NN<D>* __restrict__ nn, int n_nn,
                              const TN<D>* __restrict__ tn, int n_tn, int nk, tc::ZDesc* out_nn, tc::ZDesc* out_tn) {
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  const tc::ZDesc empty{nullptr, nullptr, nullptr, 1, 1, 1, 0, 0, 0, tc::kStore};
  if (z < n_nn * nk) {
    const NN<D> d = nn[z];
    const int64_t rows = bufs[z % nk].rows;
    out_nn[z] = (d.prec && d.n > 0 && d.k > 0)
                    ? tc::ZDesc{reinterpret_cast<const double2*>(d.A), reinterpret_cast<const double2*>(d.B),
                                reinterpret_cast<double2*>(d.C), rows, d.ldb, rows, (int)rows, d.n, d.k,
                                d.accumulate ? tc::kAdd : tc::kStore}
                    : empty;
  }
  if (z < n_tn * nk) {
    const TN<D> d = tn[z];
    const int64_t rows = bufs[z % nk].rows;
    out_tn[z] = (d.prec && d.m > 0 && d.n > 0)
                    ? tc::ZDesc{reinterpret_cast<const double2*>(d.A), reinterpret_cast<const double2*>(d.B),
                                reinterpret_cast<double2*>(d.G), rows, rows, d.ldg, d.m, d.n, (int)rows, tc::kStore}
                    : empty;
  }
}

}  // namespace dv
}  // namespace bg

#include "wide_rr.cuh"

namespace bg {
namespace dv {

// ------------------------------------------------------------------ control kernel
enum Phase : int {
  kSetup = 0,   // after H V and the Grams of the start block: factor, eigensolve
  kBegin,       // contraction at the top of an iteration
  kRefresh,     // contraction factor/eigensolve; capacity; correction rotations
  kSelect,      // drop and normalise corrections; append or stage for the repair
  kExtend,      // border the overlap factor; stage the repair
  kRepair1,     // reset to the Ritz basis; first projection Gram
  kRepair2,     // first projection; second Gram
  kRepair3,     // second projection; in-block Gram
  kRepair4,     // in-block orthonormalisation; append
  kApply,       // repair border; the apply block
  kFinish,      // border H_r, eigensolve, convergence
  kFinal,       // X = V C[:, :n]
  // with Opts::wide the phases above that factor or solve stop after posting a request
  // to the many-block kernels; these phases take their results and finish the step
  kSetupPost,
  kRefreshPost,
  kExtendPost,
  kApplyPost,
  kFinishPost,
};

constexpr int kNnSlots = 2, kTnSlots = 2, kCpSlots = 3;

template <class D>
__global__ void __launch_bounds__(kCtlThreads, 1) k_dv_ctl(int phase, Bufs<D>* __restrict__ bufs, Ctl* ctl,
                                                        NN<D>* nn, TN<D>* tn, CP<D>* cp, DynCols* dyn,
                                                        const Opts* __restrict__ opts, int nk, int gamma) {
  using X = Cx<D>;
  const Opts o = *opts;
  const int k = blockIdx.x;
  // The eigensolver's and the repair's short vectors live in shared memory (the scalar
  // QL recurrence on thread 0 reads and writes them on every rotation).
  Bufs<D> b = bufs[k];
  {
    extern __shared__ __align__(16) unsigned char dv_sm[];
    const int c = o.cap;
    D* dp = reinterpret_cast<D*>(dv_sm);
    b.off = dp;
    b.ph = dp + c;
    b.hv = dp + 2 * c;
    b.hp = dp + 3 * c;
    b.hq = dp + 4 * c;
    double* fp = reinterpret_cast<double*>(dp + 5 * c);
    b.td = fp;
    b.te = fp + c;
    b.e2 = fp + 2 * c;
    b.wu = fp + 3 * c;
    int* ip = reinterpret_cast<int*>(fp + 4 * c);
    b.order = ip;
    b.starts = ip + c;
    b.clusters = ip + 2 * c + 1;
    if (o.smem_matrices) {
      // small capacities: the eigensolver's matrices in shared memory as well
      D* mp = reinterpret_cast<D*>(ip + ((3 * c + 2 + 3) & ~3));  // 16-byte aligned
      const size_t cc = (size_t)c * c;
      b.A = mp;
      b.Y = mp + cc;
      b.Q = mp + 2 * cc;
      b.Z = reinterpret_cast<double*>(mp + 3 * cc);
    }
  }
  const int cap = o.cap, n = o.n;
  const int64_t rows = b.rows;
  __shared__ Ctl c;
  __shared__ double red[64];  // two reduction slots
  __shared__ int sh[8];
  if (threadIdx.x == 0) {
    c = ctl[k];
    for (int sl = 0; sl < kNnSlots; ++sl) nn[sl * nk + k] = NN<D>{nullptr, nullptr, nullptr, 0, 0, 0, 0};
    for (int sl = 0; sl < kTnSlots; ++sl) tn[sl * nk + k] = TN<D>{nullptr, nullptr, nullptr, 0, 0, 0};
    for (int sl = 0; sl < kCpSlots; ++sl) cp[sl * nk + k] = CP<D>{nullptr, nullptr, 0, 0};
    dyn[k] = DynCols{reinterpret_cast<const double*>(b.V), reinterpret_cast<double*>(b.HV), 0, 0};
  }
  __syncthreads();
  if (c.status != 0 && phase != kFinal) return;
  auto set_err = [&](int id) {
    if (threadIdx.x == 0) c.status = -id;
  };
  auto mirror = [&](D* M, int m0, int m1) {  // M[j][i] = conj(M[i][j]) for the new columns j in [m0, m1), i <= j
    for (int t = threadIdx.x; t < (m1 - m0) * m1; t += blockDim.x) {
      const int j = m0 + t / m1, i = t % m1;
      if (i <= j) M[j + (size_t)i * cap] = X::conj(M[i + (size_t)j * cap]);
    }
    __syncthreads();
  };
  D* Vt = b.V + (int64_t)c.m * rows;    // first free basis column
  // precision form: H Grams and rotations as tensor-core products (complex blocks)
  const int tcp = (o.tensor != 0 && sizeof(D) == sizeof(double2)) ? 1 : 0;
  // a request to the many-block reduced problem (its error bits cleared for it)
  auto request = [&](int m0, int m1, int me) {
    if (threadIdx.x == 0) {
      c.wc_m0 = m0;
      c.wc_m1 = m1;
      c.we_m = me;
      *bufs[k].werr = 0;
    }
  };
  auto clear_request = [&]() {
    if (threadIdx.x == 0) {
      c.wc_m0 = 0;
      c.wc_m1 = 0;
      c.we_m = 0;
    }
  };
  auto werr = [&]() -> int { return *(volatile int*)bufs[k].werr; };
  // capacity check, the rotations of the active Ritz vectors (after any contraction)
  auto refresh_tail = [&]() {
    if (c.m + c.nact > cap && cap < rows) {
      set_err(kErrCapacity);
      return;
    }
    const int m = c.m, na = c.nact;
    for (int t = threadIdx.x; t < m * na; t += blockDim.x) {
      const int i = t % m, j = t / m;
      b.P[i + (size_t)j * cap] = b.C[i + (size_t)b.active[j] * cap];
    }
    for (int j = threadIdx.x; j < na; j += blockDim.x) b.lam[j] = b.w[b.active[j]];
    if (threadIdx.x == 0) {
      nn[0 * nk + k] = NN<D>{b.V, b.P, b.X, cap, na, m, 0, tcp};
      nn[1 * nk + k] = NN<D>{b.HV, b.P, b.HX, cap, na, m, 0, tcp};
    }
  };
  // the repair's descriptors when the bordered factor could not be extended
  auto extend_tail = [&](bool repair) {
    const int m = c.m, kk = c.kept;
    if (threadIdx.x == 0 && repair) {
      c.repair = 1;
      c.repairs += 1;
      if (!c.need_repair) cp[0 * nk + k] = CP<D>{Vt, b.E, kk, 0};  // corrections were appended already
      nn[0 * nk + k] = NN<D>{b.V, b.C, b.X, cap, m, m, 0};
      nn[1 * nk + k] = NN<D>{b.HV, b.C, b.HX, cap, m, m, 0};
      cp[1 * nk + k] = CP<D>{b.X, b.V, m, 0};
      cp[2 * nk + k] = CP<D>{b.HX, b.HV, m, 0};
    }
  };
  auto apply_tail = [&]() {
    const int m = c.m, kk = c.kept;
    for (int i = threadIdx.x; i < n; i += blockDim.x) b.old[i] = b.w[i];
    if (threadIdx.x == 0 && kk > 0) {
      c.h_calls += 1;
      c.h_columns += kk;
      dyn[k] = DynCols{reinterpret_cast<const double*>(Vt), reinterpret_cast<double*>(b.HV + (int64_t)m * rows), kk,
                       gamma ? (kk + 1) / 2 : kk};
      tn[0 * nk + k] = TN<D>{b.V, b.HV + (int64_t)m * rows, b.Hr + (size_t)m * cap, cap, m + kk, kk, tcp};
    }
  };
  auto finish_tail = [&](int kk) {
    if (threadIdx.x == 0) {
      if (kk > 0) {
        c.m += kk;
        c.reduced_solves += 1;
      }
      int na = 0;
      double dmax = 0.0;
      for (int i = 0; i < n; ++i) {
        const double thr = (o.first_step || i < o.occupied) ? o.threshold : fmax(5.0 * o.threshold, 5e-6);
        const double change = fabs(b.w[i] - b.old[i]);
        const bool cv = change < thr;
        b.conv[i] = cv ? 1 : 0;
        if (!cv) b.active[na++] = i;
        dmax = fmax(dmax, change);
      }
      c.nact = na;
      c.iterations += 1;
      if (c.precond == BG_PRECOND_LEARNED && na > 0) {
        // TPA fallback of the learned preconditioner: the largest Ritz change has not
        // fallen below its best for kLearnedStall iterations, or half the budget is spent
        if (dmax < c.best_change) {
          c.best_change = dmax;
          c.pstall = 0;
        } else {
          ++c.pstall;
        }
        if (c.pstall >= kLearnedStall || 2 * c.iterations >= o.max_iterations) {
          c.precond = BG_PRECOND_TPA;
          c.fallbacks = 1;
        }
      }
      if (na == 0 || c.iterations == o.max_iterations) {
        c.status = 1;
      } else if (c.m + na > cap) {
        c.contract = 1;   // the reference contracts at the end of this iteration
      }
    }
  };
  auto setup_tail = [&]() {
    if (threadIdx.x == 0) {
      c.reduced_solves += 1;
      c.m = n;
      c.nact = n;
      for (int i = 0; i < n; ++i) b.active[i] = i;
    }
  };
  switch (phase) {
    case kSetup: {
      if (o.wide) {
        request(0, n, n);
        break;
      }
      if (!chol_extend(b.S, cap, b.L, 0, n, &sh[4])) {
        set_err(kErrStartDependent);
        break;
      }
      if (!eigen(b, cap, n, red, sh)) {
        set_err(kErrEigen);
        break;
      }
      setup_tail();
      break;
    }
    case kSetupPost: {
      const int we = werr();
      if (we & wide::kWErrBarrier) {
        set_err(kErrTimeout);
        break;
      }
      if (we & wide::kWErrPivot) {
        set_err(kErrStartDependent);
        break;
      }
      if (we) {
        set_err(kErrEigen);
        break;
      }
      clear_request();
      setup_tail();
      break;
    }
    case kBegin: {
      if (threadIdx.x == 0) {
        c.contract = c.contract || (c.m + c.nact > cap && c.m > n);
        if (c.contract) {
          // X = V C[:, :n], HX = HV C[:, :n] become the basis: the refresh phase exchanges
          // the buffers (no copy), so the Grams read X and HX
          nn[0 * nk + k] = NN<D>{b.V, b.C, b.X, cap, n, c.m, 0, tcp};
          nn[1 * nk + k] = NN<D>{b.HV, b.C, b.HX, cap, n, c.m, 0, tcp};
          tn[0 * nk + k] = TN<D>{b.X, b.X, b.S, cap, n, n, 0};
          tn[1 * nk + k] = TN<D>{b.X, b.HX, b.Hr, cap, n, n, tcp};
        }
      }
      break;
    }
    case kRefresh: {
      if (c.contract) {
        {
          D* t = b.V;
          b.V = b.X;
          b.X = t;
          t = b.HV;
          b.HV = b.HX;
          b.HX = t;
        }
        if (threadIdx.x == 0) {
          bufs[k].V = b.V;
          bufs[k].X = b.X;
          bufs[k].HV = b.HV;
          bufs[k].HX = b.HX;
        }
        if (o.wide) {
          request(0, n, n);
          break;
        }
        if (!chol_extend(b.S, cap, b.L, 0, n, &sh[4])) {
          set_err(kErrBasisDependent);
          break;
        }
        if (!eigen(b, cap, n, red, sh)) {
          set_err(kErrEigen);
          break;
        }
        if (threadIdx.x == 0) {
          c.contractions += 1;
          c.reduced_solves += 1;
          c.m = n;
          c.contract = 0;
        }
        __syncthreads();
      }
      if (o.wide) break;
      refresh_tail();
      break;
    }
    case kRefreshPost: {
      if (c.we_m) {  // the contraction's factor and eigensolve
        const int we = werr();
        if (we & wide::kWErrBarrier) {
          set_err(kErrTimeout);
          break;
        }
        if (we & wide::kWErrPivot) {
          set_err(kErrBasisDependent);
          break;
        }
        if (we) {
          set_err(kErrEigen);
          break;
        }
        clear_request();
        if (threadIdx.x == 0) {
          c.contractions += 1;
          c.reduced_solves += 1;
          c.m = n;
          c.contract = 0;
        }
        __syncthreads();
      }
      refresh_tail();
      break;
    }
    case kSelect: {
      if (o.tensor && o.handover > 0.0) {
        // precision form: hand over to FP64 once every active occupied band's residual is
        // below the handover residual, or when their largest residual has fallen by less
        // than 30 % in each of two iterations (the BF16x3 products' noise floor), or after
        // half of the iteration budget
        if (threadIdx.x == 0) {
          bool hand = c.iterations >= max(2, o.max_iterations / 2);
          double mx_occ = 0.0;
          for (int j = 0; j < c.nact; ++j)
            if (b.active[j] < o.occupied) mx_occ = fmax(mx_occ, b.rnorm[j]);
          if (mx_occ < o.handover * o.handover) hand = true;
          if (mx_occ < kStallFactor * c.best_res) {  // stagnation of the occupied bands
            c.stall = 0;
          } else if (++c.stall >= 2) {
            hand = true;
          }
          c.best_res = fmin(c.best_res, mx_occ);
          if (hand) c.status = 2;
        }
        __syncthreads();
        if (c.status != 0) break;
      }
      if (threadIdx.x == 0) {
        int kept = 0;
        for (int j = 0; j < c.nact; ++j) {
          const double nrm = sqrt(b.norms[j]);
          if (!isfinite(nrm)) {
            c.status = -kErrNonfiniteCorrection;
            break;
          }
          if (nrm <= 32.0 * kEps) {
            c.dropped += 1;
            continue;
          }
          b.map[kept] = j;
          b.scale[kept] = 1.0 / nrm;
          ++kept;
        }
        c.kept = kept;
        c.need_repair = (c.m + kept > cap) || kept == 0;
        c.repair = 0;
        if (c.status == 0) {
          if (!c.need_repair) {
            cp[0 * nk + k] = CP<D>{b.Er, Vt, kept, 1};
            tn[0 * nk + k] = TN<D>{b.V, Vt, b.S + (size_t)c.m * cap, cap, c.m + kept, kept};
          } else {
            cp[0 * nk + k] = CP<D>{b.Er, b.E, kept, 1};
          }
        }
      }
      break;
    }
    case kExtend: {
      const int m = c.m, kk = c.kept;
      bool repair = c.need_repair != 0;
      if (!repair) {
        mirror(b.S, m, m + kk);
        if (o.wide) {
          request(m, m + kk, 0);
          break;
        }
        if (!chol_extend(b.S, cap, b.L, m, m + kk, &sh[4])) repair = true;
      }
      if (o.wide) break;
      extend_tail(repair);
      break;
    }
    case kExtendPost: {
      bool repair = c.need_repair != 0;
      if (!repair && c.wc_m1 > c.wc_m0) {
        if (werr() & wide::kWErrBarrier) {
          set_err(kErrTimeout);
          break;
        }
        repair = werr() != 0;
      }
      clear_request();
      extend_tail(repair);
      break;
    }
    case kRepair1: {
      if (!c.repair) break;
      const int m = c.m;
      for (int t = threadIdx.x; t < m * m; t += blockDim.x) {
        const int i = t % m, j = t / m;
        const bool dg = i == j;
        b.S[i + (size_t)j * cap] = dg ? X::one() : X::zero();
        b.L[i + (size_t)j * cap] = dg ? X::one() : X::zero();
        b.Hr[i + (size_t)j * cap] = dg ? X::from_real(b.w[i]) : X::zero();
        b.C[i + (size_t)j * cap] = dg ? X::one() : X::zero();
      }
      if (threadIdx.x == 0 && c.kept > 0) tn[0 * nk + k] = TN<D>{b.V, b.E, b.P, cap, m, c.kept};
      break;
    }
    case kRepair2:
    case kRepair3: {
      if (!c.repair || c.kept == 0) break;
      const int m = c.m, kk = c.kept;
      for (int t = threadIdx.x; t < m * kk; t += blockDim.x) {
        const int i = t % m, j = t / m;
        b.P[i + (size_t)j * cap] = X::neg(b.P[i + (size_t)j * cap]);
      }
      if (threadIdx.x == 0) {
        nn[0 * nk + k] = NN<D>{b.V, b.P, b.E, cap, kk, m, 1};
        // the in-block Gram goes to the global A (another kernel writes it)
        tn[0 * nk + k] = phase == kRepair2 ? TN<D>{b.V, b.E, b.P, cap, m, kk} : TN<D>{b.E, b.E, bufs[k].A, cap, kk, kk};
      }
      break;
    }
    case kRepair4: {
      if (!c.repair || c.kept == 0) break;
      const int kraw = c.kept;
      const D* G = bufs[k].A;
      D* Qc = b.P;   // orthonormal combinations, column q of kept j
      D* q = b.hv;
      D* dots = b.hp;
      D* t = b.hq;
      if (threadIdx.x == 0) sh[5] = 0;
      __syncthreads();
      for (int j = 0; j < kraw; ++j) {
        const int nkeep = sh[5];
        // dots with the kept combinations: q_c^H G e_j
        for (int cc = threadIdx.x; cc < nkeep; cc += blockDim.x) {
          D acc = X::zero();
          for (int a = 0; a < kraw; ++a) acc = X::add(acc, X::mul(X::conj(Qc[a + (size_t)cc * cap]), G[a + (size_t)j * cap]));
          dots[cc] = acc;
        }
        __syncthreads();
        for (int a = threadIdx.x; a < kraw; a += blockDim.x) {
          D v = a == j ? X::one() : X::zero();
          for (int cc = 0; cc < nkeep; ++cc) v = X::sub(v, X::mul(dots[cc], Qc[a + (size_t)cc * cap]));
          q[a] = v;
        }
        __syncthreads();
        double part = 0.0;
        for (int a = threadIdx.x; a < kraw; a += blockDim.x) {
          D acc = X::zero();
          for (int bb = 0; bb < kraw; ++bb) acc = X::add(acc, X::mul(G[a + (size_t)bb * cap], q[bb]));
          t[a] = acc;
          part += X::dot_re(q[a], acc);
        }
        const double len = sqrt(fmax(block_sum(part, red), 0.0));
        if (!(len > kDependence)) {
          if (threadIdx.x == 0) c.dropped += 1;
          __syncthreads();
          continue;
        }
        for (int a = threadIdx.x; a < kraw; a += blockDim.x) Qc[a + (size_t)nkeep * cap] = X::div(q[a], len);
        __syncthreads();
        if (threadIdx.x == 0) sh[5] = nkeep + 1;
        __syncthreads();
      }
      if (threadIdx.x == 0) {
        const int kk = min(sh[5], cap - c.m);
        c.kept = kk;
        if (kk > 0) {
          nn[0 * nk + k] = NN<D>{b.E, Qc, b.Er, cap, kk, kraw, 0};
          cp[0 * nk + k] = CP<D>{b.Er, Vt, kk, 0};
          tn[0 * nk + k] = TN<D>{b.V, Vt, b.S + (size_t)c.m * cap, cap, c.m + kk, kk};
        }
      }
      break;
    }
    case kApply: {
      const int m = c.m, kk = c.kept;
      if (c.repair && kk > 0) {
        mirror(b.S, m, m + kk);
        if (o.wide) {
          request(m, m + kk, 0);
          break;
        }
        if (!chol_extend(b.S, cap, b.L, m, m + kk, &sh[4])) {
          set_err(kErrRepairDependent);
          break;
        }
      }
      if (o.wide) break;
      apply_tail();
      break;
    }
    case kApplyPost: {
      if (c.wc_m1 > c.wc_m0) {
        if (werr() & wide::kWErrBarrier) {
          set_err(kErrTimeout);
          break;
        }
        if (werr()) {
          set_err(kErrRepairDependent);
          break;
        }
        clear_request();
      }
      apply_tail();
      break;
    }
    case kFinish: {
      const int kk = c.kept;
      if (kk > 0) {
        mirror(b.Hr, c.m, c.m + kk);
        if (o.wide) {
          request(0, 0, c.m + kk);
          break;
        }
        if (!eigen(b, cap, c.m + kk, red, sh)) {
          set_err(kErrEigen);
          break;
        }
      }
      if (o.wide) break;
      finish_tail(kk);
      break;
    }
    case kFinishPost: {
      if (c.we_m) {
        if (werr() & wide::kWErrBarrier) {
          set_err(kErrTimeout);
          break;
        }
        if (werr()) {
          set_err(kErrEigen);
          break;
        }
        clear_request();
      }
      finish_tail(c.kept);
      break;
    }
    case kFinal: {
      if (c.status < 0) break;
      if (threadIdx.x == 0) {
        nn[0 * nk + k] = NN<D>{b.V, b.C, b.X, cap, n, c.m, 0, tcp};
        if (o.want_hx) nn[1 * nk + k] = NN<D>{b.HV, b.C, b.HX, cap, n, c.m, 0, tcp};
      }
      break;
    }
    default:
      break;
  }
  __syncthreads();
  if (threadIdx.x == 0) ctl[k] = c;
}

// ------------------------------------------------------------------ start and outputs
// Per-k pointers of a solve's inputs and outputs (device array, one entry per k point).
struct IoPtrs {
  const void* start;     // device start block (rows x n), or null (copied from the host)
  const double* diag;    // device diagonal, or null
  void* vectors;         // device output block, or null (copied to the host)
  const int* err;        // the operator's device error word
  const void* start_hx;  // device H of the start block (kept from an earlier solve), or null
  void* vectors_hx;      // device output H X, or null
};

// Zero S, H_r, L, C of every k point and copy its start block and diagonal from device
// pointers: one launch instead of six stream operations per k point.  blockIdx.y = k.
template <class D>
__global__ void k_dv_init(const Bufs<D>* __restrict__ bufs, const IoPtrs* __restrict__ io, int n, int cap) {
  const int k = blockIdx.y;
  const Bufs<D>& b = bufs[k];
  const int64_t cc = (int64_t)cap * cap, rn = (int64_t)b.rows * n;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t t0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  for (int64_t t = t0; t < 4 * cc; t += stride) {
    D* m = t < cc ? b.S : (t < 2 * cc ? b.Hr : (t < 3 * cc ? b.L : b.C));
    m[t % cc] = Cx<D>::zero();
  }
  const IoPtrs p = io[k];
  if (p.start) {
    const D* src = static_cast<const D*>(p.start);
    for (int64_t t = t0; t < rn; t += stride) b.V[t] = src[t];
  }
  if (p.start_hx) {
    const D* src = static_cast<const D*>(p.start_hx);
    for (int64_t t = t0; t < rn; t += stride) b.HV[t] = src[t];
  }
  if (p.diag)
    for (int64_t t = t0; t < b.rows; t += stride) const_cast<double*>(b.diag)[t] = p.diag[t];
}

// Outputs of every k point: X to the device output block, and the eigenvalues,
// convergence flags and the operator's error word gathered for one read by the host
// (out: nk n values, then nk n flags and nk error words as doubles).  blockIdx.y = k.
template <class D>
__global__ void k_dv_out(const Bufs<D>* __restrict__ bufs, const IoPtrs* __restrict__ io, int n, int nk,
                         double* __restrict__ out) {
  const int k = blockIdx.y;
  const Bufs<D>& b = bufs[k];
  const IoPtrs p = io[k];
  const int64_t rn = (int64_t)b.rows * n;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t t0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p.vectors) {
    D* dst = static_cast<D*>(p.vectors);
    for (int64_t t = t0; t < rn; t += stride) dst[t] = b.X[t];
  }
  if (p.vectors_hx) {
    D* dst = static_cast<D*>(p.vectors_hx);
    for (int64_t t = t0; t < rn; t += stride) dst[t] = b.HX[t];
  }
  if (blockIdx.x == 0) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      out[(int64_t)k * n + i] = b.w[i];
      out[(int64_t)nk * n + (int64_t)k * n + i] = (double)b.conv[i];
    }
    if (threadIdx.x == 0) out[2 * (int64_t)nk * n + k] = (double)*p.err;
  }
}

// ------------------------------------------------------------------ host side
template <class T>
struct DevOf;
template <>
struct DevOf<double> {
  using type = double;
};
template <>
struct DevOf<std::complex<double>> {
  using type = double2;
};

const char* error_text(int id) {
  switch (id) {
    case kErrStartDependent: return "reference Davidson start is numerically dependent";
    case kErrBasisDependent: return "reference Davidson basis is numerically dependent";
    case kErrNonfiniteCorrection: return "nonfinite reference correction";
    case kErrCapacity: return "capacity cannot hold the active correction block; use at least 2*bands";
    case kErrRepairDependent: return "reference overlap remains dependent after repair";
    case kErrEigen: return "reference reduced eigensolve failed";
    case kErrTimeout: return "a grid barrier of the many-block reduced problem gave up";
    default: return "reference Davidson failed";
  }
}

template <class T>
class KsetSolver {
 public:
  using D = typename DevOf<T>::type;
  KsetSolver(bg_kset* ks, int n, int cap, bool wide) : ks_(ks), nk_((int)ks->ops.size()), wide_(wide) {
    o_.n = n;
    o_.cap = cap;
    o_.smem_matrices = small(cap) ? 1 : 0;
    o_.wide = wide ? 1 : 0;
  }
  bool matches(int n, int cap, bool wide) const { return o_.n == n && o_.cap == cap && wide_ == wide; }
  // Per-call options (threshold, occupied, first_step, iterations, preconditioner).
  // The captured iteration holds the apply's kernels, so each apply precision keeps a
  // graph of its own.
  void set_options(const Opts& o, bool graph) {
    o_ = o;
    o_.smem_matrices = small(o.cap) ? 1 : 0;
    o_.wide = wide_ ? 1 : 0;
    want_graph_ = graph;
  }
  ~KsetSolver() {
    tcnl_.release();
    for (int p = 0; p < 3; ++p) {
      if (exec_[p]) cudaGraphExecDestroy(exec_[p]);
      if (graph_[p]) cudaGraphDestroy(graph_[p]);
    }
    for (void* p : dev_) cudaFree(p);
    if (h_ctl_) cudaFreeHost(h_ctl_);
    if (h_out_) cudaFreeHost(h_out_);
    if (h_io_) cudaFreeHost(h_io_);
  }
  int run(const double* const* start, const double* const* diagonal, int32_t ptr_kind, double* const* values,
          double* const* vectors, int32_t* const* converged, bg_davidson_stats* stats,
          const double* const* start_hx = nullptr, double* const* vectors_hx = nullptr);
  const std::string& error() const { return err_; }
  int64_t launches() const { return launches_; }

 private:
  bg_kset* ks_;
  int nk_;
  bool wide_ = false;
  // precision form: the solver's own tensor-core nonlocal buffers and the descriptors and
  // split-K workspace of its tensor-core Davidson products
  TcNl tcnl_;
  tc::ZDesc* d_tcnn_ = nullptr;
  tc::ZDesc* d_tctn_ = nullptr;
  unsigned char* tc_work_ = nullptr;
  int* tc_err_ = nullptr;
  int tc_ks_ = 1;
  bool tc_ready_ = false;
  unsigned* d_bar_ = nullptr;   // grid barrier of the cooperative launches
  double* d_wpart_ = nullptr;   // their per-block partial sums
  int coop_blocks_ = 0;
  Opts o_;
  bool want_graph_ = true;
  bool prepared_ = false;
  bool graph_tried_[3] = {false, false, false};   // by precision (0 FP64, 1 FP32, 2 tensor)
  Opts* d_opts_ = nullptr;
  cudaStream_t s_ = nullptr;
  std::vector<void*> dev_;
  std::vector<Bufs<D>> hb_;
  Bufs<D>* d_bufs_ = nullptr;
  Ctl* d_ctl_ = nullptr;
  Ctl* h_ctl_ = nullptr;
  IoPtrs* d_io_ = nullptr;
  IoPtrs* h_io_ = nullptr;
  double* d_out_ = nullptr;
  double* h_out_ = nullptr;
  NN<D>* d_nn_ = nullptr;
  TN<D>* d_tn_ = nullptr;
  CP<D>* d_cp_ = nullptr;
  DynCols* d_dyn_ = nullptr;
  const D** d_dense_ = nullptr;
  int ksplit_ = 1;
  int64_t slot_elems_ = 0;
  int max_rows_ = 0;
  std::vector<CallArgs> args_;
  std::vector<int64_t> cols_;
  cudaGraph_t graph_[3] = {nullptr, nullptr, nullptr};
  cudaGraphExec_t exec_[3] = {nullptr, nullptr, nullptr};
  int64_t per_iteration_[3] = {0, 0, 0};
  int64_t launches_ = 0;
  std::string err_;

  template <class P>
  int alloc(P** p, size_t count) {
    void* q = nullptr;
    if (cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(P)) != cudaSuccess) {
      err_ = "cudaMalloc failed";
      return BG_ENOMEM;
    }
    dev_.push_back(q);
    *p = static_cast<P*>(q);
    return BG_OK;
  }
  int cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return BG_OK;
    err_ = std::string(what) + ": " + cudaGetErrorString(e);
    return BG_EDEVICE;
  }
  static size_t vec_smem(int cap) {
    return (size_t)cap * (5 * sizeof(D) + 4 * sizeof(double)) + sizeof(int) * (size_t)((3 * cap + 2 + 3) & ~3);
  }
  static size_t mat_smem(int cap) { return (size_t)cap * cap * (3 * sizeof(D) + sizeof(double)); }
  // A, Y, Q and Z join the vectors in shared memory when all fit in 200 KB.
  static bool small(int cap) { return vec_smem(cap) + mat_smem(cap) <= 200 * 1024; }
  size_t ctl_smem() const { return vec_smem(o_.cap) + (o_.smem_matrices ? mat_smem(o_.cap) : 0); }
  int64_t ctl(int phase) {
    k_dv_ctl<D><<<nk_, kCtlThreads, ctl_smem(), s_>>>(phase, d_bufs_, d_ctl_, d_nn_, d_tn_, d_cp_, d_dyn_, d_opts_,
                                                     nk_, ks_->gamma);
    return 1;
  }
  int64_t nn(int nslots) {
    const dim3 grid((unsigned)((o_.cap + 63) / 64), (unsigned)((max_rows_ + 63) / 64), (unsigned)(nslots * nk_));
    k_dv_nn<D><<<grid, 256, tiles::nn64m_smem_bytes<D>(), s_>>>(d_bufs_, d_nn_, nk_);
    if (!tensor_products()) return 1;
    k_dv_tc_descs<D><<<1, 128, 0, s_>>>(d_bufs_, d_nn_, nslots, d_tn_, 0, nk_, d_tcnn_, d_tctn_);
    return 2 + tc::launch_zgemm(tc::kNN, d_tcnn_, nslots * nk_, max_rows_, o_.cap, o_.cap, 1, false, tc_work_,
                                tc_err_, s_);
  }
  bool tensor_products() const { return o_.tensor && sizeof(D) == sizeof(double2) && tc_ready_; }
  int64_t tn(int nslots) {
    const unsigned t = (unsigned)((o_.cap + 47) / 48);
    k_dv_tn<D><<<dim3(t, t, (unsigned)(nslots * nk_ * ksplit_)), 256, tiles::tn48m_smem_bytes<D>(), s_>>>(
        d_bufs_, d_tn_, nk_, ksplit_, slot_elems_);
    const unsigned blocks = (unsigned)std::min<int64_t>(((int64_t)o_.cap * o_.cap + 255) / 256, 64);
    k_dv_tn_sum<D><<<dim3(blocks, 1, (unsigned)(nslots * nk_)), 256, 0, s_>>>(d_bufs_, d_tn_, nk_, ksplit_,
                                                                              slot_elems_);
    if (!tensor_products()) return 2;
    k_dv_tc_descs<D><<<1, 128, 0, s_>>>(d_bufs_, d_nn_, 0, d_tn_, nslots, nk_, d_tcnn_, d_tctn_);
    return 3 + tc::launch_zgemm(tc::kTN, d_tctn_, nslots * nk_, o_.cap, o_.cap, max_rows_, tc_ks_, false, tc_work_,
                                tc_err_, s_);
  }
  // Buffers of the precision form (once, before any capture).
  int prepare_tensor() {
    if (tc_ready_ || sizeof(D) != sizeof(double2)) return BG_OK;
    int rc;
    if ((rc = cuda(tc::prepare_zgemm(), "tensor-core product attributes"))) return rc;
    const int slots = std::max(kNnSlots, kTnSlots);
    tc_ks_ = tc::tn_ksplit_tuned(kTnSlots * nk_, o_.cap, o_.cap, max_rows_);
    if ((rc = alloc(&d_tcnn_, (size_t)slots * nk_)) || (rc = alloc(&d_tctn_, (size_t)slots * nk_)) ||
        (rc = alloc(&tc_work_, std::max(tc::workspace_bytes(tc::kTN, kTnSlots * nk_, o_.cap, o_.cap, max_rows_,
                                                             tc_ks_, false),
                                         tc::workspace_bytes(tc::kNN, kNnSlots * nk_, max_rows_, o_.cap, o_.cap, 1,
                                                             false)))) ||
        (rc = alloc(&tc_err_, 1)))
      return rc;
    if ((rc = cuda(cudaMemset(tc_err_, 0, sizeof(int)), "tensor error word"))) return rc;
    if (!ks_->gamma && ks_->shape.nproj > 0 && ensure_nonlocal_tc(&tcnl_, nk_, ks_->shape.nproj, o_.n, max_rows_)) {
      err_ = "tensor-core nonlocal buffers";
      return BG_ENOMEM;
    }
    tc_ready_ = true;
    return BG_OK;
  }
  int64_t cp(int slot0, int nslots) {
    const int64_t span = 256 * kCopyUnroll;
    const dim3 grid((unsigned)std::min<int64_t>((max_rows_ + span - 1) / span, 64), (unsigned)o_.cap,
                    (unsigned)(nslots * nk_));
    k_dv_copy<D><<<grid, 256, 0, s_>>>(d_bufs_, d_cp_ + (size_t)slot0 * nk_, nk_);
    return 1;
  }
  int64_t corr() {
    k_dv_corrections<D><<<dim3((unsigned)o_.n, (unsigned)nk_), 256, 0, s_>>>(
        d_bufs_, d_ctl_, d_opts_, static_cast<const __nv_bfloat16*>(ks_->ctx->learned));
    return 1;
  }
  // Many-block reduced problem (wide_rr.cuh): extension of the factor, then the
  // eigensolve; each launch returns at once for k points without a request.
  int64_t wchol() {
    return wide::launch_chol<D>(d_bufs_, d_ctl_, nk_, o_.cap, coop_blocks_, d_bar_, s_);
  }
  int64_t weig() {
    return wide::launch_eig<D>(d_bufs_, d_ctl_, nk_, o_.cap, coop_blocks_, d_bar_, d_wpart_, s_);
  }
  int64_t apply() {
    if (ks_->dense) {
      const dim3 grid((unsigned)((max_rows_ + 63) / 64), (unsigned)((o_.n + 31) / 32), (unsigned)nk_);
      k_dv_dense<D><<<grid, 128, 0, s_>>>(d_dense_, d_bufs_, d_dyn_);
      return 1;
    }
    return enqueue_range(ks_, 0, nk_, args_.data(), cols_.data(), s_, nullptr,
                         o_.tensor ? BG_PREC_TENSOR : (o_.fp32 ? BG_PREC_FP32 : BG_PREC_FP64), &tcnl_);
  }
  int64_t iteration() {
    int64_t l = 0;
    l += ctl(kBegin) + nn(2) + tn(2);
    l += ctl(kRefresh);
    if (wide_) l += wchol() + weig() + ctl(kRefreshPost);
    l += nn(2) + corr();
    l += ctl(kSelect) + cp(0, 1) + tn(1);
    l += ctl(kExtend);
    if (wide_) l += wchol() + ctl(kExtendPost);
    l += cp(0, 1) + nn(2) + cp(1, 2);
    l += ctl(kRepair1) + tn(1);
    l += ctl(kRepair2) + nn(1) + tn(1);
    l += ctl(kRepair3) + nn(1) + tn(1);
    l += ctl(kRepair4) + nn(1) + cp(0, 1) + tn(1);
    l += ctl(kApply);
    if (wide_) l += wchol() + ctl(kApplyPost);
    l += apply() + tn(1);
    l += ctl(kFinish);
    if (wide_) l += weig() + ctl(kFinishPost);
    return l;
  }
  int prepare();
  int poll(bool* all_done) {
    int rc = cuda(cudaMemcpyAsync(h_ctl_, d_ctl_, sizeof(Ctl) * nk_, cudaMemcpyDeviceToHost, s_), "poll");
    if (!rc) rc = cuda(cudaStreamSynchronize(s_), "Davidson iteration");
    if (rc) return rc;
    *all_done = true;
    for (int k = 0; k < nk_; ++k) {
      if (h_ctl_[k].status < 0) {
        err_ = std::string(error_text(-h_ctl_[k].status)) + " (k point " + std::to_string(k) + ")";
        return BG_EINVAL;
      }
      if (h_ctl_[k].status == 0) *all_done = false;
    }
    return BG_OK;
  }
};

template <class T>
int KsetSolver<T>::prepare() {
  const int n = o_.n, cap = o_.cap;
  int rc;
  hb_.resize(nk_);
  max_rows_ = 0;
  for (int k = 0; k < nk_; ++k) max_rows_ = std::max<int>(max_rows_, (int)ks_->ops[k]->rows);
  // Gram row slices: about four 256-thread blocks per SM over all (tile, k) pairs
  const int64_t tiles = (int64_t)((cap + 47) / 48) * ((cap + 47) / 48);
  ksplit_ = (int)std::max<int64_t>(1, std::min<int64_t>((4 * 148 + tiles * nk_ - 1) / (tiles * nk_), 32));
  ksplit_ = (int)std::max<int64_t>(1, std::min<int64_t>(ksplit_, (max_rows_ + 127) / 128));
  slot_elems_ = (int64_t)ksplit_ * cap * cap;
  const size_t cc = (size_t)cap * cap;
  for (int k = 0; k < nk_; ++k) {
    Bufs<D>& b = hb_[k];
    const size_t rc_ = (size_t)ks_->ops[k]->rows * cap;
    b.rows = (int)ks_->ops[k]->rows;
    if ((rc = alloc(&b.V, rc_)) || (rc = alloc(&b.HV, rc_)) || (rc = alloc(&b.X, rc_)) || (rc = alloc(&b.HX, rc_)) ||
        (rc = alloc(&b.E, rc_)) || (rc = alloc(&b.Er, rc_)) || (rc = alloc(&b.S, cc)) || (rc = alloc(&b.Hr, cc)) ||
        (rc = alloc(&b.L, cc)) || (rc = alloc(&b.C, cc)) || (rc = alloc(&b.A, cc)) || (rc = alloc(&b.Y, cc)) ||
        (rc = alloc(&b.P, cc)) || (rc = alloc(&b.Q, cc)) || (rc = alloc(&b.Z, cc)) || (rc = alloc(&b.w, cap)) ||
        (rc = alloc(&b.old, cap)) || (rc = alloc(&b.lam, cap)) || (rc = alloc(&b.norms, cap)) ||
        (rc = alloc(&b.scale, cap)) || (rc = alloc(&b.td, cap)) || (rc = alloc(&b.te, cap)) ||
        (rc = alloc(&b.rnorm, cap)) ||
        (rc = alloc(&b.off, cap)) || (rc = alloc(&b.ph, cap)) || (rc = alloc(&b.hv, cap)) || (rc = alloc(&b.hp, cap)) ||
        (rc = alloc(&b.hq, cap)) || (rc = alloc(&b.active, cap)) || (rc = alloc(&b.map, cap)) ||
        (rc = alloc(&b.conv, cap)) || (rc = alloc(&b.order, cap)) || (rc = alloc(&b.part, 2 * (size_t)slot_elems_)) ||
        false)
      return rc;
    double* dg = nullptr;
    if ((rc = alloc(&dg, b.rows))) return rc;
    b.diag = dg;
    if (wide_) {
      if ((rc = alloc(&b.LT, cc)) || (rc = alloc(&b.lu, 4 * cc)) || (rc = alloc(&b.werr, 1)) ||
          (rc = alloc(&b.wmeta, 8)) || (rc = alloc(&b.wimeta, 8)) || (rc = alloc(&b.e2, cap)) ||
          (rc = alloc(&b.wu, cap)) || (rc = alloc(&b.starts, cap + 1)) || (rc = alloc(&b.clusters, cap + 1)))
        return rc;
    }
  }
  if (wide_) {
    if ((rc = wide::prepare<D>(cap, &coop_blocks_, &err_))) return rc;
    if ((rc = alloc(&d_bar_, 2)) || (rc = alloc(&d_wpart_, 2 * (size_t)coop_blocks_))) return rc;
  }
  if ((rc = alloc(&d_bufs_, nk_)) || (rc = alloc(&d_ctl_, nk_)) || (rc = alloc(&d_nn_, (size_t)kNnSlots * nk_)) ||
      (rc = alloc(&d_tn_, (size_t)kTnSlots * nk_)) || (rc = alloc(&d_cp_, (size_t)kCpSlots * nk_)) ||
      (rc = alloc(&d_dyn_, nk_)) || (rc = alloc(&d_opts_, 1)))
    return rc;
  if ((rc = cuda(cudaMallocHost(&h_ctl_, sizeof(Ctl) * nk_), "cudaMallocHost"))) return rc;
  if ((rc = alloc(&d_io_, nk_)) || (rc = alloc(&d_out_, (size_t)nk_ * (2 * n + 1)))) return rc;
  if ((rc = cuda(cudaMallocHost(&h_io_, sizeof(IoPtrs) * nk_), "cudaMallocHost")) ||
      (rc = cuda(cudaMallocHost(&h_out_, sizeof(double) * nk_ * (2 * n + 1)), "cudaMallocHost")))
    return rc;
  if ((rc = cuda(cudaFuncSetAttribute((const void*)k_dv_ctl<D>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)ctl_smem()),
                 "cudaFuncSetAttribute")) ||
      (rc = cuda(cudaFuncSetAttribute((const void*)k_dv_tn<D>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)tiles::tn48m_smem_bytes<D>()),
                 "cudaFuncSetAttribute")) ||
      (rc = cuda(cudaFuncSetAttribute((const void*)k_dv_nn<D>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)tiles::nn64m_smem_bytes<D>()),
                 "cudaFuncSetAttribute")))
    return rc;
  if (ks_->dense) {
    std::vector<const D*> hd(nk_);
    for (int k = 0; k < nk_; ++k) hd[k] = reinterpret_cast<const D*>(ks_->ops[k]->dense);
    if ((rc = alloc(&d_dense_, nk_))) return rc;
    if ((rc = cuda(cudaMemcpy(d_dense_, hd.data(), sizeof(const D*) * nk_, cudaMemcpyHostToDevice), "upload")))
      return rc;
  }
  if ((rc = cuda(cudaMemcpy(d_bufs_, hb_.data(), sizeof(Bufs<D>) * nk_, cudaMemcpyHostToDevice), "upload")))
    return rc;
  args_.assign(nk_, CallArgs{});
  cols_.assign(nk_, n);
  for (int k = 0; k < nk_; ++k) {
    CallArgs& a = args_[k];
    const int64_t dpc = ks_->gamma ? hb_[k].rows : 2 * (int64_t)hb_[k].rows;
    a.x = reinterpret_cast<const double*>(hb_[k].V);
    a.y = reinterpret_cast<double*>(hb_[k].HV);
    a.ldx = a.ldy = dpc;
    a.cols = n;
    a.units = ks_->gamma ? (n + 1) / 2 : n;
    a.dyn = d_dyn_ + k;
  }
  prepared_ = true;
  return BG_OK;
}

template <class T>
int KsetSolver<T>::run(const double* const* start, const double* const* diagonal, int32_t ptr_kind,
                       double* const* values, double* const* vectors, int32_t* const* converged,
                       bg_davidson_stats* stats, const double* const* start_hx, double* const* vectors_hx) {
  const int n = o_.n, cap = o_.cap;
  int rc;
  const bool kept = start_hx != nullptr && ptr_kind == BG_PTR_DEVICE;
  o_.want_hx = vectors_hx != nullptr && ptr_kind == BG_PTR_DEVICE ? 1 : 0;
  s_ = ks_->stream;
  launches_ = 0;
  if (!prepared_ && (rc = prepare())) return rc;
  if (o_.tensor && (rc = prepare_tensor())) return rc;
  // the pinned pointer table may still feed a copy of the previous solve
  if ((rc = cuda(cudaStreamSynchronize(s_), "start"))) return rc;
  for (int k = 0; k < nk_; ++k) {
    const bool dev = ptr_kind == BG_PTR_DEVICE;
    h_io_[k] = IoPtrs{dev ? start[k] : nullptr, dev ? diagonal[k] : nullptr, dev ? vectors[k] : nullptr,
                      ks_->ops[k]->t.err, kept ? start_hx[k] : nullptr, o_.want_hx ? vectors_hx[k] : nullptr};
    if (!dev) {  // host inputs: one copy each
      const Bufs<D>& b = hb_[k];
      if ((rc = cuda(cudaMemcpyAsync(b.V, start[k], sizeof(D) * (size_t)b.rows * n, cudaMemcpyHostToDevice, s_),
                     "copy in")) ||
          (rc = cuda(cudaMemcpyAsync(const_cast<double*>(b.diag), diagonal[k], sizeof(double) * b.rows,
                                     cudaMemcpyHostToDevice, s_), "copy in")))
        return rc;
    }
  }
  if ((rc = cuda(cudaMemcpyAsync(d_io_, h_io_, sizeof(IoPtrs) * nk_, cudaMemcpyHostToDevice, s_), "upload")))
    return rc;
  k_dv_init<D><<<dim3(64, nk_), 256, 0, s_>>>(d_bufs_, d_io_, n, cap);
  launches_ += 1;
  if ((rc = cuda(cudaMemcpyAsync(d_opts_, &o_, sizeof(Opts), cudaMemcpyHostToDevice, s_), "upload"))) return rc;
  // start: H V and the Grams of the start block, descriptors written from the host
  std::vector<Ctl> c0(nk_);
  std::vector<DynCols> dy(nk_);
  std::vector<TN<D>> t0((size_t)kTnSlots * nk_);
  for (int k = 0; k < nk_; ++k) {
    Ctl& c = c0[k];
    std::memset(&c, 0, sizeof c);
    c.m = n;
    c.nact = n;
    c.h_calls = kept ? 0 : 1;   // a kept H V needs no apply
    c.h_columns = kept ? 0 : n;
    c.best_res = 1e300;
    c.precond = o_.preconditioner;
    c.best_change = 1e300;
    const Bufs<D>& b = hb_[k];
    dy[k] = DynCols{reinterpret_cast<const double*>(b.V), reinterpret_cast<double*>(b.HV), n,
                    ks_->gamma ? (n + 1) / 2 : n};
    t0[k] = TN<D>{b.V, b.V, b.S, cap, n, n};
    t0[(size_t)nk_ + k] = TN<D>{b.V, b.HV, b.Hr, cap, n, n, (o_.tensor && sizeof(D) == sizeof(double2)) ? 1 : 0};
  }
  if ((rc = cuda(cudaMemcpyAsync(d_ctl_, c0.data(), sizeof(Ctl) * nk_, cudaMemcpyHostToDevice, s_), "upload")) ||
      (rc = cuda(cudaMemcpyAsync(d_dyn_, dy.data(), sizeof(DynCols) * nk_, cudaMemcpyHostToDevice, s_), "upload")) ||
      (rc = cuda(cudaMemcpyAsync(d_tn_, t0.data(), sizeof(TN<D>) * t0.size(), cudaMemcpyHostToDevice, s_), "upload")))
    return rc;
  if (wide_ && (rc = cuda(cudaMemsetAsync(d_bar_, 0, 2 * sizeof(unsigned), s_), "barrier"))) return rc;
  launches_ += (kept ? 0 : apply()) + tn(2) + ctl(kSetup);
  if (wide_) launches_ += wchol() + weig() + ctl(kSetupPost);
  bool done = false;
  if ((rc = poll(&done))) return rc;
  // iterations: one captured graph replayed until every k point has finished
  const int gp = o_.tensor ? 2 : (o_.fp32 ? 1 : 0);
  if (want_graph_ && !graph_tried_[gp]) {
    graph_tried_[gp] = true;
    cudaStreamCaptureStatus st;
    if (cudaStreamIsCapturing(s_, &st) == cudaSuccess && st == cudaStreamCaptureStatusNone &&
        cudaStreamBeginCapture(s_, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
      const int64_t per = iteration();
      if (cudaStreamEndCapture(s_, &graph_[gp]) == cudaSuccess && graph_[gp] &&
          cudaGraphInstantiate(&exec_[gp], graph_[gp], 0) == cudaSuccess)
        per_iteration_[gp] = per;
      else if (exec_[gp]) {
        cudaGraphExecDestroy(exec_[gp]);
        exec_[gp] = nullptr;
      }
    }
    cudaGetLastError();
  }
  const bool graph_ok = want_graph_ && exec_[gp] != nullptr;
  for (int it = 0; it < o_.max_iterations && !done; ++it) {
    if (graph_ok) {
      if ((rc = cuda(cudaGraphLaunch(exec_[gp], s_), "cudaGraphLaunch"))) return rc;
      launches_ += per_iteration_[gp];
    } else {
      launches_ += iteration();
    }
    if ((rc = cuda(cudaGetLastError(), "Davidson launch"))) return rc;
    if ((rc = poll(&done))) return rc;
  }
  // X = V C[:, :n]; outputs
  launches_ += ctl(kFinal) + nn(o_.want_hx ? 2 : 1);
  if ((rc = poll(&done))) return rc;
  // contractions exchange V and X (and HV and HX) on the device: refresh the host mirror
  if ((rc = cuda(cudaMemcpy(hb_.data(), d_bufs_, sizeof(Bufs<D>) * nk_, cudaMemcpyDeviceToHost), "buffers")))
    return rc;
  k_dv_out<D><<<dim3(64, nk_), 256, 0, s_>>>(d_bufs_, d_io_, n, nk_, d_out_);
  launches_ += 1;
  const size_t outn = (size_t)nk_ * (2 * n + 1);
  if ((rc = cuda(cudaMemcpyAsync(h_out_, d_out_, sizeof(double) * outn, cudaMemcpyDeviceToHost, s_), "copy out")))
    return rc;
  if (ptr_kind != BG_PTR_DEVICE)
    for (int k = 0; k < nk_; ++k)
      if ((rc = cuda(cudaMemcpyAsync(vectors[k], hb_[k].X, sizeof(D) * (size_t)hb_[k].rows * n,
                                     cudaMemcpyDeviceToHost, s_), "copy out")))
        return rc;
  if ((rc = cuda(cudaStreamSynchronize(s_), "copy out"))) return rc;
  for (int k = 0; k < nk_; ++k) {
    const Ctl& c = h_ctl_[k];
    bg_davidson_stats st{};
    for (int i = 0; i < n; ++i) {
      values[k][i] = h_out_[(size_t)k * n + i];
      converged[k][i] = c.iterations > 0 ? (int)h_out_[(size_t)nk_ * n + (size_t)k * n + i] : 0;
      st.converged_count += converged[k][i];
    }
    st.iterations = c.iterations;
    st.reduced_solves = c.reduced_solves;
    st.h_calls = c.h_calls;
    st.h_columns = c.h_columns;
    st.repairs = c.repairs;
    st.contractions = c.contractions;
    st.dropped = c.dropped;
    st.fallbacks = c.fallbacks;
    if (stats) stats[k] = st;
  }
  // the tensor-core products' pipelines (bounded waits) must not have given up
  if (o_.tensor && tc_ready_) {
    int words[2] = {0, 0};
    if ((rc = cuda(cudaMemcpy(&words[0], tc_err_, sizeof(int), cudaMemcpyDeviceToHost), "tensor error word")))
      return rc;
    if (tcnl_.err && (rc = cuda(cudaMemcpy(&words[1], tcnl_.err, sizeof(int), cudaMemcpyDeviceToHost), "tensor error word")))
      return rc;
    if (words[0] || words[1]) {
      cudaMemset(tc_err_, 0, sizeof(int));
      if (tcnl_.err) cudaMemset(tcnl_.err, 0, sizeof(int));
      err_ = "a tensor-core product's pipeline wait gave up";
      return BG_ETIMEOUT;
    }
  }
  // a non-finite block met by the applies
  for (int k = 0; k < nk_; ++k) {
    if (h_out_[2 * (size_t)nk_ * n + k] != 0.0) {
      cudaMemsetAsync(ks_->ops[k]->t.err, 0, sizeof(int), s_);
      cudaStreamSynchronize(s_);
      err_ = "non-finite block in a Davidson apply (k point " + std::to_string(k) + ")";
      return BG_ENONFINITE;
    }
  }
  return BG_OK;
}

// Generalised Hermitian eigenproblem H C = S C diag(w) of one m x m pencil through the
// many-block path of the batched Davidson (wide_rr.cuh): the Cholesky factor of S with the
// pivot rule, then A = L^-1 H L^-H, its eigenpairs and C = L^-H Y.
template <class D>
int reduced_eigh(int m, const double* S, const double* H, double* w, double* C, double* ms, std::string* err) {
  std::vector<void*> mem;
  auto alloc = [&](auto** p, size_t count) -> bool {
    void* q = nullptr;
    if (cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(**p)) != cudaSuccess) return false;
    mem.push_back(q);
    *p = static_cast<std::remove_reference_t<decltype(**p)>*>(q);
    return true;
  };
  struct Free {
    std::vector<void*>* m;
    ~Free() {
      for (void* p : *m) cudaFree(p);
    }
  } guard{&mem};
  const int cap = m;
  const size_t cc = (size_t)cap * cap;
  Bufs<D> b{};
  bool ok = alloc(&b.S, cc) && alloc(&b.Hr, cc) && alloc(&b.L, cc) && alloc(&b.C, cc) && alloc(&b.A, cc) &&
            alloc(&b.Y, cc) && alloc(&b.Q, cc) && alloc(&b.Z, cc) && alloc(&b.LT, cc) && alloc(&b.lu, 4 * cc) &&
            alloc(&b.w, cap) && alloc(&b.td, cap) && alloc(&b.te, cap) && alloc(&b.e2, cap) && alloc(&b.wu, cap) &&
            alloc(&b.off, cap) && alloc(&b.ph, cap) && alloc(&b.hp, cap) && alloc(&b.hq, cap) && alloc(&b.hv, cap) &&
            alloc(&b.starts, cap + 1) &&
            alloc(&b.clusters, cap + 1) && alloc(&b.order, cap) && alloc(&b.werr, 1) && alloc(&b.wmeta, 8) &&
            alloc(&b.wimeta, 8);
  Bufs<D>* d_b = nullptr;
  Ctl* d_c = nullptr;
  unsigned* bar = nullptr;
  double* part = nullptr;
  int blocks = 0;
  ok = ok && alloc(&d_b, 1) && alloc(&d_c, 1) && alloc(&bar, 2);
  if (!ok) {
    *err = "cudaMalloc failed";
    return BG_ENOMEM;
  }
  int rc = wide::prepare<D>(cap, &blocks, err);
  if (rc) return rc;
  if (!alloc(&part, 2 * (size_t)blocks)) {
    *err = "cudaMalloc failed";
    return BG_ENOMEM;
  }
  Ctl c{};
  c.wc_m0 = 0;
  c.wc_m1 = m;
  c.we_m = m;
  cudaStream_t s = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  if (e == cudaSuccess) e = cudaMemcpyAsync(b.S, S, sizeof(D) * cc, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(b.Hr, H, sizeof(D) * cc, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(b.L, 0, sizeof(D) * cc, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(b.werr, 0, sizeof(int), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned), s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_b, &b, sizeof b, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_c, &c, sizeof c, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaEventRecord(e0, s);
  if (e == cudaSuccess) {
    wide::launch_chol<D>(d_b, d_c, 1, cap, blocks, bar, s);
    wide::launch_eig<D>(d_b, d_c, 1, cap, blocks, bar, part, s);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaEventRecord(e1, s);
  int werr = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&werr, b.werr, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  float t = 0.0f;
  if (e == cudaSuccess && ms) e = cudaEventElapsedTime(&t, e0, e1);
  if (ms) *ms = t;
  if (e == cudaSuccess && !werr) {
    e = cudaMemcpy(w, b.w, sizeof(double) * m, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(C, b.C, sizeof(D) * cc, cudaMemcpyDeviceToHost);
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (s) cudaStreamDestroy(s);
  if (e != cudaSuccess) {
    *err = std::string("reduced eigensolve: ") + cudaGetErrorString(e);
    return BG_EDEVICE;
  }
  if (werr & wide::kWErrBarrier) {
    *err = "reduced eigensolve: a grid barrier gave up";
    return BG_ETIMEOUT;
  }
  if (werr & wide::kWErrPivot) {
    *err = "overlap is numerically dependent (pivot rule)";
    return BG_ESHAPE;
  }
  if (werr) {
    *err = "non-finite reduced matrix";
    return BG_ENONFINITE;
  }
  return BG_OK;
}

}  // namespace dv
}  // namespace bg

using namespace bg;
using namespace bg::dv;

namespace {
int kset_solve(bg_kset* ks, const double* const* start, const double* const* start_hx, const double* const* diagonal,
               const bg_davidson_options* options, int32_t ptr_kind, double* const* eigenvalues,
               double* const* eigenvectors, double* const* eigenvectors_hx, int32_t* const* converged,
               bg_davidson_stats* stats) {
  if (!ks) return fail(nullptr, BG_EINVAL, "null k-point set");
  bg_ctx* ctx = ks->ctx;
  if (!start || !diagonal || !options || !eigenvalues || !eigenvectors || !converged)
    return fail(ctx, BG_EINVAL, "null argument");
  if (ptr_kind != BG_PTR_HOST && ptr_kind != BG_PTR_DEVICE) return fail(ctx, BG_EINVAL, "pointer kind");
  if ((start_hx || eigenvectors_hx) && ptr_kind != BG_PTR_DEVICE)
    return fail(ctx, BG_EINVAL, "kept H X blocks are device blocks");
  for (int k = 0; k < (int)ks->ops.size(); ++k)
    if ((start_hx && !start_hx[k]) || (eigenvectors_hx && !eigenvectors_hx[k]))
      return fail(ctx, BG_EINVAL, "null per-k H X block");
  const bg_davidson_options o = *options;
  const int nk = (int)ks->ops.size();
  const int64_t n = o.bands;
  int64_t cap = o.capacity == 0 ? 2 * n : o.capacity;
  bool bad = n <= 0 || o.occupied > n || o.occupied < 0 || o.max_iterations <= 0 || !std::isfinite(o.threshold) ||
             o.threshold <= 0.0 || o.preconditioner < BG_PRECOND_SMOOTH || o.preconditioner > BG_PRECOND_LEARNED;
  for (int k = 0; k < nk && !bad; ++k) {
    const bg_op* op = ks->ops[k];
    const int64_t rows = op->rows;
    // crates/dft-solvers/src/ref_davidson.rs:133-146, per k point
    const int64_t capk = std::min<int64_t>(cap, rows);
    bad = n > rows || capk < std::min<int64_t>(2 * n, rows) || n > op->cap;
    cap = std::min(cap, capk);
  }
  if (bad || cap > 1536)
    return fail(ctx, BG_EINVAL, "reference Davidson dimensions/threshold (bands must fit every operator's capacity)");
  if (o.preconditioner == BG_PRECOND_LEARNED && !ctx->learned)
    return fail(ctx, BG_EINVAL, "learned preconditioner requested but no network was set (bg_learned_set)");
  for (int k = 0; k < nk; ++k) {
    if (!start[k] || !diagonal[k] || !eigenvalues[k] || !eigenvectors[k] || !converged[k])
      return fail(ctx, BG_EINVAL, "null per-k argument");
    if (!ks->ops[k]->has_epoch) return fail(ctx, BG_EEPOCH, "potential was never set");
    if (ptr_kind == BG_PTR_HOST) {
      const size_t per = ks->gamma ? 1 : 2;
      const int64_t rows = ks->ops[k]->rows;
      for (size_t i = 0; i < (size_t)rows * n * per; ++i)
        if (!std::isfinite(start[k][i])) return fail(ctx, BG_ENONFINITE, "reference Davidson start not finite");
      for (int64_t i = 0; i < rows; ++i)
        if (!std::isfinite(diagonal[k][i])) return fail(ctx, BG_ENONFINITE, "reference Davidson diagonal not finite");
    }
  }
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
  if (o.apply_precision != BG_PREC_FP64 && o.apply_precision != BG_PREC_FP32 && o.apply_precision != BG_PREC_TENSOR)
    return fail(ctx, BG_EINVAL, "unsupported apply precision");
  if (o.apply_precision != BG_PREC_FP64 && (ks->dense || !fp32_supported(ks->g)))
    return fail(ctx, BG_EINVAL, "the FP32 apply needs a cubic grid of 25, 45, 54, 60, 72 or 108 points");
  Opts op{(int)n, (int)cap, (int)o.occupied, o.first_step ? 1 : 0, o.max_iterations, o.threshold, o.preconditioner, 0,
          o.apply_precision != BG_PREC_FP64 ? 1 : 0};
  op.tensor = o.apply_precision == BG_PREC_TENSOR ? 1 : 0;
  op.handover = op.tensor ? kHandoverResidual : 0.0;
  const bool graph = (o.flags & 1) == 0;
  // the reduced problem on many blocks for capacities 129 .. 1152 (flags bit 1 forces it,
  // bit 2 keeps the one-block control kernel)
  const bool wide = (o.flags & 2) != 0 || (cap > 128 && cap <= wide::kMaxCap && (o.flags & 4) == 0);
  int rc;
  if (o.apply_precision != BG_PREC_FP64)  // the FP32 potential copies, on the set's stream
    for (bg_op* kop : ks->ops)
      if ((rc = ensure_potential_float(kop, ks->stream))) return rc;
  std::string err;
  int64_t launches = 0;
  // The solver (device work arrays, descriptors and the captured iteration graph) lives
  // on the set and is reused while bands and capacity stay the same.
  auto solve = [&](auto* tag) -> int {
    using S = std::remove_pointer_t<decltype(tag)>;
    S* s = static_cast<S*>(ks->dv_cache);
    if (s && !s->matches(op.n, op.cap, wide)) {
      ks->dv_free(ks->dv_cache);
      ks->dv_cache = nullptr;
      s = nullptr;
    }
    if (!s) {
      s = new S(ks, op.n, op.cap, wide);
      ks->dv_cache = s;
      ks->dv_free = [](void* p) { delete static_cast<S*>(p); };
    }
    s->set_options(op, graph);
    int r = s->run(start, diagonal, ptr_kind, eigenvalues, eigenvectors, converged, stats, start_hx, eigenvectors_hx);
    err = s->error();
    launches = s->launches();
    if (r != BG_OK || !op.tensor) return r;
    // precision form: when the tensor phase converged every band by the Davidson's own
    // Ritz-change criterion at a loose threshold (kTensorOnlyThreshold) it stands;
    // otherwise (a handover, or bands left unconverged) the FP64 phase runs from its Ritz
    // vectors and judges convergence in FP64
    bool all = op.threshold >= kTensorOnlyThreshold;
    for (int k = 0; k < nk && all; ++k)
      for (int64_t i = 0; i < n && all; ++i) all = converged[k][i] != 0;
    if (all) {
      if (stats)
        for (int k = 0; k < nk; ++k) stats[k].tensor_iterations = stats[k].iterations;
      return r;
    }
    std::vector<bg_davidson_stats> first(stats ? (size_t)nk : 0);
    if (stats) std::copy(stats, stats + nk, first.begin());
    Opts o64 = op;
    o64.fp32 = 0;
    o64.tensor = 0;
    o64.handover = 0.0;
    s->set_options(o64, graph);
    r = s->run(eigenvectors, diagonal, ptr_kind, eigenvalues, eigenvectors, converged, stats, nullptr,
               eigenvectors_hx);
    err = s->error();
    launches += s->launches();
    if (stats)
      for (int k = 0; k < nk; ++k) {
        bg_davidson_stats& st = stats[k];
        const bg_davidson_stats& f = first[k];
        st.tensor_iterations = f.iterations;
        st.iterations += f.iterations;
        st.reduced_solves += f.reduced_solves;
        st.h_calls += f.h_calls;
        st.h_columns += f.h_columns;
        st.repairs += f.repairs;
        st.contractions += f.contractions;
        st.dropped += f.dropped;
      }
    return r;
  };
  if (ks->gamma)
    rc = solve(static_cast<KsetSolver<double>*>(nullptr));
  else
    rc = solve(static_cast<KsetSolver<std::complex<double>>*>(nullptr));
  ks->launches += launches;
  if (rc != BG_OK) return fail(ctx, rc, err.empty() ? "reference Davidson failed" : err);
  return BG_OK;
}
}  // namespace

extern "C" int bg_kset_davidson_solve(bg_kset* ks, const double* const* start, const double* const* diagonal,
                                      const bg_davidson_options* options, int32_t ptr_kind, double* const* eigenvalues,
                                      double* const* eigenvectors, int32_t* const* converged,
                                      bg_davidson_stats* stats) {
  return kset_solve(ks, start, nullptr, diagonal, options, ptr_kind, eigenvalues, eigenvectors, nullptr, converged,
                    stats);
}

extern "C" int bg_kset_davidson_solve_hx(bg_kset* ks, const double* const* start, const double* const* start_hx,
                                         const double* const* diagonal, const bg_davidson_options* options,
                                         double* const* eigenvalues, double* const* eigenvectors,
                                         double* const* eigenvectors_hx, int32_t* const* converged,
                                         bg_davidson_stats* stats) {
  return kset_solve(ks, start, start_hx, diagonal, options, BG_PTR_DEVICE, eigenvalues, eigenvectors, eigenvectors_hx,
                    converged, stats);
}

extern "C" int bg_reduced_eigh(bg_ctx* ctx, int64_t m, int32_t is_complex, const double* s, const double* h,
                               double* eigenvalues, double* vectors, double* device_ms) {
  if (!ctx) return fail(nullptr, BG_EINVAL, "null context");
  if (!s || !h || !eigenvalues || !vectors) return fail(ctx, BG_EINVAL, "null argument");
  if (m < 1 || m > wide::kMaxCap) return fail(ctx, BG_ESHAPE, "reduced problem size must be in [1, 1152]");
  const size_t n = (size_t)m * m * (is_complex ? 2 : 1);
  for (size_t i = 0; i < n; ++i)
    if (!std::isfinite(s[i]) || !std::isfinite(h[i])) return fail(ctx, BG_ENONFINITE, "non-finite pencil");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
  std::string err;
  const int rc = is_complex ? reduced_eigh<double2>((int)m, s, h, eigenvalues, vectors, device_ms, &err)
                            : reduced_eigh<double>((int)m, s, h, eigenvalues, vectors, device_ms, &err);
  if (rc != BG_OK) return fail(ctx, rc, err);
  return BG_OK;
}
