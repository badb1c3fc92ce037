// Small dense linear algebra of the Davidson reduced problem (host, FP64), templated
// on double (real Gamma ORC rows) and std::complex<double> (k points).
//
// * cholesky_extend: bordered Cholesky S = L L^H of the leading m0 x m0 block
//   extended to m columns, with the reference's pivot rule: every new column's
//   squared pivot over its overlap diagonal must be at least eps / 1e-12
//   (crates/dft-solvers/src/lean_davidson.rs:62-70, 228-240).
// * heev: Hermitian eigensolver, eigenvalues ascending: Householder reduction to a
//   real symmetric tridiagonal matrix (a unitary diagonal scaling removes the phases
//   of the off-diagonal), implicit QL iteration with Wilkinson shifts on the
//   tridiagonal, back-transformation of the eigenvectors.  Matrices are column-major
//   with leading dimension ld.
#pragma once
#include <algorithm>
#include <cmath>
#include <complex>
#include <limits>
#include <numeric>
#include <vector>

namespace bg {
namespace dense {

using cplx = std::complex<double>;

inline double re(double x) { return x; }
inline double re(const cplx& x) { return x.real(); }
inline double conj(double x) { return x; }
inline cplx conj(const cplx& x) { return std::conj(x); }
inline double abs2(double x) { return x * x; }
inline double abs2(const cplx& x) { return std::norm(x); }

constexpr double kPivotRatioMin = std::numeric_limits<double>::epsilon() / 1e-12;

// Extend the lower Cholesky factor L (columns 0..m0-1 valid) to columns m0..m-1 of S.
// Returns false when a pivot ratio falls below kPivotRatioMin or is not finite.
template <class T>
bool cholesky_extend(const T* S, int ld, T* L, int m0, int m) {
  for (int j = m0; j < m; ++j) {
    // row j of L: L[j][k] = (S[j][k] - sum_{p<k} L[j][p] conj(L[k][p])) / L[k][k]
    for (int k = 0; k < j; ++k) {
      T x = S[j + (size_t)k * ld];
      for (int p = 0; p < k; ++p) x -= L[j + (size_t)p * ld] * conj(L[k + (size_t)p * ld]);
      L[j + (size_t)k * ld] = x / re(L[k + (size_t)k * ld]);
    }
    double d = re(S[j + (size_t)j * ld]);
    for (int p = 0; p < j; ++p) d -= abs2(L[j + (size_t)p * ld]);
    const double ratio = d / re(S[j + (size_t)j * ld]);
    if (!(ratio >= kPivotRatioMin) || !std::isfinite(ratio)) return false;
    L[j + (size_t)j * ld] = T(std::sqrt(d));
    for (int i = 0; i < j; ++i) L[i + (size_t)j * ld] = T(0);
  }
  return true;
}

// B <- L^{-1} B (L lower, m x m; B m x n).
template <class T>
void solve_lower(const T* L, int ldl, T* B, int ldb, int m, int n) {
  for (int c = 0; c < n; ++c) {
    T* b = B + (size_t)c * ldb;
    for (int i = 0; i < m; ++i) {
      T x = b[i];
      for (int k = 0; k < i; ++k) x -= L[i + (size_t)k * ldl] * b[k];
      b[i] = x / re(L[i + (size_t)i * ldl]);
    }
  }
}

// B <- L^{-H} B.
template <class T>
void solve_lower_adjoint(const T* L, int ldl, T* B, int ldb, int m, int n) {
  for (int c = 0; c < n; ++c) {
    T* b = B + (size_t)c * ldb;
    for (int i = m - 1; i >= 0; --i) {
      T x = b[i];
      for (int k = i + 1; k < m; ++k) x -= conj(L[k + (size_t)i * ldl]) * b[k];
      b[i] = x / re(L[i + (size_t)i * ldl]);
    }
  }
}

// Implicit QL on the symmetric tridiagonal (d diagonal, e[i] between i and i+1,
// e[n-1] ignored); Z (n x n, column-major, ld n) accumulates the rotations.
inline bool tridiagonal_ql(std::vector<double>& d, std::vector<double>& e, std::vector<double>& Z, int n) {
  if (n == 0) return true;
  e[n - 1] = 0.0;
  for (int l = 0; l < n; ++l) {
    int iter = 0;
    int m;
    do {
      for (m = l; m < n - 1; ++m) {
        const double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
        if (std::fabs(e[m]) <= std::numeric_limits<double>::epsilon() * dd) break;
      }
      if (m != l) {
        if (iter++ == 60) return false;
        double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
        double r = std::hypot(g, 1.0);
        g = d[m] - d[l] + e[l] / (g + (g >= 0.0 ? r : -r));
        double s = 1.0, c = 1.0, p = 0.0;
        int i;
        for (i = m - 1; i >= l; --i) {
          double f = s * e[i];
          const double b = c * e[i];
          r = std::hypot(f, g);
          e[i + 1] = r;
          if (r == 0.0) {
            d[i + 1] -= p;
            e[m] = 0.0;
            break;
          }
          s = f / r;
          c = g / r;
          g = d[i + 1] - p;
          r = (d[i] - g) * s + 2.0 * c * b;
          p = s * r;
          d[i + 1] = g + p;
          g = c * r - b;
          for (int k = 0; k < n; ++k) {
            f = Z[k + (size_t)(i + 1) * n];
            Z[k + (size_t)(i + 1) * n] = s * Z[k + (size_t)i * n] + c * f;
            Z[k + (size_t)i * n] = c * Z[k + (size_t)i * n] - s * f;
          }
        }
        if (r == 0.0 && i >= l) continue;
        d[l] -= p;
        e[l] = g;
        e[m] = 0.0;
      }
    } while (m != l);
  }
  return true;
}

// Eigen-decomposition of the Hermitian n x n matrix A (column-major, ld): w ascending,
// V (ld n) the eigenvectors.  A is overwritten.  Returns false on a QL failure or a
// non-finite input.
template <class T>
bool heev(T* A, int lda, int n, double* w, T* V, int ldv) {
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i)
      if (!std::isfinite(re(A[i + (size_t)j * lda])) || !std::isfinite(std::abs(A[i + (size_t)j * lda]))) return false;
  // symmetrise the rounding of the input
  for (int j = 0; j < n; ++j) {
    A[j + (size_t)j * lda] = T(re(A[j + (size_t)j * lda]));
    for (int i = j + 1; i < n; ++i) {
      const T avg = (A[i + (size_t)j * lda] + conj(A[j + (size_t)i * lda])) * 0.5;
      A[i + (size_t)j * lda] = avg;
      A[j + (size_t)i * lda] = conj(avg);
    }
  }
  std::vector<T> Q((size_t)n * n, T(0));
  for (int i = 0; i < n; ++i) Q[i + (size_t)i * n] = T(1);
  std::vector<T> v(n), p(n), q(n);
  std::vector<T> off(n > 0 ? n : 1, T(0));
  for (int k = 0; k + 2 < n; ++k) {
    const int L = n - k - 1;
    T* x = A + (k + 1) + (size_t)k * lda;
    double xn2 = 0.0;
    for (int i = 0; i < L; ++i) xn2 += abs2(x[i]);
    const double xn = std::sqrt(xn2);
    if (xn == 0.0) {
      off[k] = T(0);
      continue;
    }
    const double ax0 = std::abs(x[0]);
    const T phase = ax0 > 0.0 ? x[0] / ax0 : T(1);
    const T alpha = -phase * xn;
    for (int i = 0; i < L; ++i) v[i] = x[i];
    v[0] -= alpha;
    double vn2 = 0.0;
    for (int i = 0; i < L; ++i) vn2 += abs2(v[i]);
    if (vn2 == 0.0) {
      off[k] = x[0];
      continue;
    }
    const double beta = 2.0 / vn2;
    // p = beta B v, B = A[k+1:, k+1:]
    for (int i = 0; i < L; ++i) {
      T s = T(0);
      for (int j = 0; j < L; ++j) s += A[(k + 1 + i) + (size_t)(k + 1 + j) * lda] * v[j];
      p[i] = beta * s;
    }
    T vp = T(0);
    for (int i = 0; i < L; ++i) vp += conj(v[i]) * p[i];
    const double K = 0.5 * beta * re(vp);
    for (int i = 0; i < L; ++i) q[i] = p[i] - K * v[i];
    for (int j = 0; j < L; ++j)
      for (int i = 0; i < L; ++i)
        A[(k + 1 + i) + (size_t)(k + 1 + j) * lda] -= v[i] * conj(q[j]) + q[i] * conj(v[j]);
    off[k] = alpha;
    for (int i = 0; i < L; ++i) {
      x[i] = T(0);
      A[k + (size_t)(k + 1 + i) * lda] = T(0);
    }
    // Q <- Q H on columns k+1..n-1
    for (int r = 0; r < n; ++r) {
      T s = T(0);
      for (int j = 0; j < L; ++j) s += Q[r + (size_t)(k + 1 + j) * n] * v[j];
      s *= beta;
      for (int j = 0; j < L; ++j) Q[r + (size_t)(k + 1 + j) * n] -= s * conj(v[j]);
    }
  }
  if (n >= 2) off[n - 2] = A[(n - 1) + (size_t)(n - 2) * lda];
  // phases: T_real = D^H T D with s_0 = 1, s_{k+1} = s_k off_k / |off_k|
  std::vector<T> s(n, T(1));
  std::vector<double> d(n), e(n, 0.0);
  for (int k = 0; k < n; ++k) d[k] = re(A[k + (size_t)k * lda]);
  for (int k = 0; k + 1 < n; ++k) {
    const double a = std::abs(off[k]);
    e[k] = a;
    s[k + 1] = a > 0.0 ? s[k] * (off[k] / a) : s[k];
  }
  std::vector<double> Z((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) Z[i + (size_t)i * n] = 1.0;
  if (!tridiagonal_ql(d, e, Z, n)) return false;
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return d[a] < d[b]; });
  for (int c = 0; c < n; ++c) {
    const int src = order[c];
    w[c] = d[src];
    for (int r = 0; r < n; ++r) {
      T acc = T(0);
      for (int k = 0; k < n; ++k) acc += Q[r + (size_t)k * n] * (s[k] * Z[k + (size_t)src * n]);
      V[r + (size_t)c * ldv] = acc;
    }
  }
  return true;
}

}  // namespace dense
}  // namespace bg
