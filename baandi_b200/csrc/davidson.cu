// Block Davidson of the reference SCF (FP64): subspace products on the GPU, the small
// reduced problem (bordered Cholesky, Hermitian eigensolve) on the host.
//
// Restates crates/dft-solvers/src/ref_davidson.rs:117-366 (real Gamma ORC rows) and
// crates/dft-solvers/src/ref_davidson_complex.rs:641-1110 (complex), one rank:
//   setup     V = start, HV = H V, S = V^H V, L L^H = S (pivot rule), H_r = V^H H V,
//             A = L^-1 H_r L^-H, A Y = Y diag(lambda), C = L^-H Y
//   iterate   contraction when m + active > cap (V <- V C[:, :n], HV <- HV C[:, :n],
//             refreshed S, H_r, factor and eigensolve);
//             corrections E_j = (HX_j - lambda_j X_j) / d(h, lambda_j) with
//             X = V C[:, active], HX = HV C[:, active] and the smooth denominator
//             d = (2 max(x, 1) + 1 / (sqrt(1 + z^2) + z)) / 4, x = 2 (h - lambda),
//             z = |x - 1| (ref_davidson.rs:418-422, ref_davidson/stream.rs:16-67);
//             corrections of norm <= 32 eps are dropped, the others normalised;
//             append, border S, extend the factor; a rejected pivot triggers the
//             repair (basis rotated to its Ritz vectors, corrections projected out
//             of it twice, in-block orthonormalisation with the 1e-12 dependence
//             floor); H E, border H_r, eigensolve;
//             Ritz-change convergence |lambda_i - lambda_i,old| < threshold_i with
//             the occupied / empty band thresholds of ref_davidson.rs:70-76.
//   finish    X = V C[:, :n], eigenvalues lambda_0..n-1.
// The reference's ideal-reset shortcut after a contraction is replaced by the measured
// refresh it falls back to; the iterates differ only in rounding.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <string>
#include <memory>
#include <vector>

#include "blas_dev.cuh"
#include "gemm_tiles.cuh"
#include "dense_host.h"
#include "op_internal.h"

namespace bg {
namespace {

constexpr double kEps = 2.220446049250313e-16;
constexpr double kDependence = 1e-12;  // crates/dft-numerics/src/linalg.rs:12

// ------------------------------------------------------------------ kernels
// E[:, j] = correction of band j (correction_column, preconditioner `kind`; kind 3 reads
// the learned network's BF16 parameters `net`); norms2[j] = |E[:, j]|^2.
template <class D, bool LEARNED>
__global__ void __launch_bounds__(256) k_corrections(const D* __restrict__ X, const D* __restrict__ HX, int64_t ld,
                                                     const double* __restrict__ diag, const double* __restrict__ lambda,
                                                     D* __restrict__ E, double* __restrict__ norms2, int64_t rows,
                                                     int kind, const __nv_bfloat16* __restrict__ net) {
  __shared__ double red[256];
  __shared__ float wnet[LEARNED ? learned::kParams : 1];
  if constexpr (LEARNED) learned::load_params(net, wnet);
  const int j = blockIdx.x;
  const double n2 =
      correction_column<D, LEARNED>(X + j * ld, HX + j * ld, diag, lambda[j], kind, rows, E + j * ld, red, wnet);
  if (threadIdx.x == 0) norms2[j] = n2;
}

// out[:, c] = scale[c] * in[:, map[c]]
template <class D>
__global__ void k_pick_scale(const D* __restrict__ in, int64_t ld, const int* __restrict__ map,
                             const double* __restrict__ scale, D* __restrict__ out, int64_t rows) {
  const int c = blockIdx.y;
  const D* src = in + (int64_t)map[c] * ld;
  D* dst = out + (int64_t)c * ld;
  const double s = scale[c];
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x)
    dst[r] = Arith<D>::scale(s, src[r]);
}

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

// ------------------------------------------------------------------ solver
template <class T>
class Solver {
 public:
  using D = typename DevOf<T>::type;

  Solver(bg_op* op, int n, int cap, const bg_davidson_options& o) : op_(op), n_(n), cap_(cap), o_(o) {
    rows_ = op->rows;
    s_ = op->stream;
    kind_ = o.preconditioner;
  }

  int run(const T* start, const double* diagonal, double* values_out, T* vectors_out, int32_t* converged,
          bg_davidson_stats* st);
  const std::string& error() const { return err_; }

 private:
  bg_op* op_;
  int64_t rows_;
  int n_, cap_;
  bg_davidson_options o_;
  int kind_;  // preconditioner in use: the learned one gives way to TPA when the solve stalls
  cudaStream_t s_;
  size_t next_ = 0;  // next arena slot
  D *V_ = nullptr, *HV_ = nullptr, *X_ = nullptr, *HX_ = nullptr, *E_ = nullptr, *Er_ = nullptr, *HE_ = nullptr;
  D *part_ = nullptr, *small_ = nullptr, *coef_ = nullptr;
  double *diag_ = nullptr, *lam_ = nullptr, *norms_ = nullptr, *scale_ = nullptr;
  int* map_ = nullptr;
  size_t part_elems_ = 0;
  std::vector<T> S_, Hr_, L_, C_;  // cap x cap, ld cap
  std::vector<double> values_, old_;
  bg_davidson_stats stats_{};
  std::string err_;
  static constexpr int kStallSteps = 5;
  double best_change_ = INFINITY;
  int stalled_ = 0;

  double band_threshold(int i) const {
    return (o_.first_step || i < o_.occupied) ? o_.threshold : std::max(5.0 * o_.threshold, 5e-6);
  }
  // The next work array from the operator's arena (allocated, or enlarged, only when this
  // solve needs more than an earlier one did).
  template <class P>
  int alloc(P** p, size_t count) {
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(P);
    std::vector<std::unique_ptr<DevBuf>>& arena = op_->dv_arena;
    if (next_ == arena.size()) arena.push_back(std::make_unique<DevBuf>());
    DevBuf& b = *arena[next_++];
    if (b.bytes < bytes) {
      if (b.p) cudaFree(b.p);
      b.p = nullptr;
      b.bytes = 0;
      if (cudaMalloc(&b.p, bytes) != cudaSuccess) return BG_ENOMEM;
      b.bytes = bytes;
    }
    *p = static_cast<P*>(b.p);
    return BG_OK;
  }
  int check(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      err_ = std::string(what) + ": " + cudaGetErrorString(e);
      return BG_EDEVICE;
    }
    return BG_OK;
  }
  int sync(const char* what) {
    cudaError_t e = cudaStreamSynchronize(s_);
    if (e != cudaSuccess) {
      err_ = std::string(what) + ": " + cudaGetErrorString(e);
      return BG_EDEVICE;
    }
    return BG_OK;
  }
  // G (m x k, host, ld ldg) = A[:, 0:m]^H B[:, 0:k] (device, ld rows)
  int gram(const D* A, int m, const D* B, int k, T* G, int ldg);
  // C[:, 0:k] = A[:, 0:m] Coef (m x k host, ld m); accumulate adds
  int rotate(const D* A, int m, const T* coef, int k, D* Cout, bool accumulate = false);
  int apply(const D* x, D* y, int k);
  int refresh(int m);
  int eigen(int m);
  int corrections(const std::vector<int>& active, int m, const double* diag_host, int* kept);
  int repair(int m, int* kept);
  int contract(int m);
};

template <class T>
int Solver<T>::gram(const D* A, int m, const D* B, int k, T* G, int ldg) {
  if (m == 0 || k == 0) return BG_OK;
  const int64_t tiles = (int64_t)((m + 31) / 32) * ((k + 31) / 32);
  int64_t ks = std::max<int64_t>(1, (8 * 148 + tiles - 1) / tiles);
  ks = std::min<int64_t>(ks, (rows_ + 255) / 256);
  ks = std::max<int64_t>(1, std::min<int64_t>(ks, (int64_t)(part_elems_ / ((size_t)m * k))));
  int64_t chunk = (rows_ + ks - 1) / ks;
  chunk = ((chunk + 31) / 32) * 32;
  ks = (rows_ + chunk - 1) / chunk;
  const dim3 grid((m + 31) / 32, (k + 31) / 32, (unsigned)ks);
  k_gemm_tn<D><<<grid, 64, 0, s_>>>(A, rows_, B, rows_, part_, m, k, rows_, chunk);
  k_sum_parts<D><<<(unsigned)std::min<int64_t>(((int64_t)m * k + 255) / 256, 4096), 256, 0, s_>>>(part_, (int)ks, m, k,
                                                                                                  small_, m);
  std::vector<T> h((size_t)m * k);
  cudaMemcpyAsync(h.data(), small_, sizeof(T) * h.size(), cudaMemcpyDeviceToHost, s_);
  int rc = sync("gram");
  if (rc) return rc;
  for (int j = 0; j < k; ++j)
    for (int i = 0; i < m; ++i) G[i + (size_t)j * ldg] = h[i + (size_t)j * m];
  return check("gram");
}

template <class T>
int Solver<T>::rotate(const D* A, int m, const T* coef, int k, D* Cout, bool accumulate) {
  if (k == 0) return BG_OK;
  cudaMemcpyAsync(coef_, coef, sizeof(T) * (size_t)m * k, cudaMemcpyHostToDevice, s_);
  const dim3 grid((unsigned)((rows_ + 63) / 64), (k + 31) / 32);
  k_gemm_nn<D><<<grid, 128, 0, s_>>>(A, rows_, coef_, m, Cout, rows_, rows_, k, m, accumulate ? 1 : 0);
  int rc = sync("rotate");  // coef host buffer is reused by the caller
  return rc ? rc : check("rotate");
}

template <class T>
int Solver<T>::apply(const D* x, D* y, int k) {
  if (k == 0) return BG_OK;
  stats_.h_calls += 1;
  stats_.h_columns += k;
  int rc = bg_op_apply_block(op_, reinterpret_cast<const double*>(x), reinterpret_cast<double*>(y), rows_, k,
                             BG_PTR_DEVICE, o_.apply_precision);
  if (rc != BG_OK) {
    err_ = "operator apply failed: " + op_->ctx->error;
    return rc;
  }
  return bg_op_sync(op_);
}

// S and H_r of the first m columns, their factor and the reduced eigensolve.
template <class T>
int Solver<T>::refresh(int m) {
  int rc = gram(V_, m, V_, m, S_.data(), cap_);
  if (!rc) rc = gram(V_, m, HV_, m, Hr_.data(), cap_);
  if (rc) return rc;
  if (!dense::cholesky_extend(S_.data(), cap_, L_.data(), 0, m)) {
    err_ = "reference Davidson basis is numerically dependent";
    return BG_EINVAL;
  }
  return eigen(m);
}

template <class T>
int Solver<T>::eigen(int m) {
  std::vector<T> A((size_t)m * m), Y((size_t)m * m);
  for (int j = 0; j < m; ++j)
    for (int i = 0; i < m; ++i) A[i + (size_t)j * m] = Hr_[i + (size_t)j * cap_];
  std::vector<T> Lm((size_t)m * m);
  for (int j = 0; j < m; ++j)
    for (int i = 0; i < m; ++i) Lm[i + (size_t)j * m] = L_[i + (size_t)j * cap_];
  // A <- L^-1 A L^-H
  dense::solve_lower(Lm.data(), m, A.data(), m, m, m);
  std::vector<T> At((size_t)m * m);
  for (int j = 0; j < m; ++j)
    for (int i = 0; i < m; ++i) At[i + (size_t)j * m] = dense::conj(A[j + (size_t)i * m]);
  dense::solve_lower(Lm.data(), m, At.data(), m, m, m);
  for (int j = 0; j < m; ++j)
    for (int i = 0; i < m; ++i) A[i + (size_t)j * m] = dense::conj(At[j + (size_t)i * m]);
  std::vector<double> w(m);
  stats_.reduced_solves += 1;
  if (!dense::heev(A.data(), m, m, w.data(), Y.data(), m)) {
    err_ = "reference reduced eigensolve failed";
    return BG_EINVAL;
  }
  dense::solve_lower_adjoint(Lm.data(), m, Y.data(), m, m, m);
  for (int j = 0; j < m; ++j)
    for (int i = 0; i < m; ++i) C_[i + (size_t)j * cap_] = Y[i + (size_t)j * m];
  values_.assign(w.begin(), w.end());
  return BG_OK;
}

// Corrections of the active bands into E_ (normalised, compacted); *kept columns.
template <class T>
int Solver<T>::corrections(const std::vector<int>& active, int m, const double* diag_host, int* kept) {
  (void)diag_host;
  const int k = (int)active.size();
  std::vector<T> cs((size_t)m * k);
  std::vector<double> lam(k);
  for (int j = 0; j < k; ++j) {
    for (int i = 0; i < m; ++i) cs[i + (size_t)j * m] = C_[i + (size_t)active[j] * cap_];
    lam[j] = values_[active[j]];
  }
  int rc = rotate(V_, m, cs.data(), k, X_);
  if (!rc) rc = rotate(HV_, m, cs.data(), k, HX_);
  if (rc) return rc;
  cudaMemcpyAsync(lam_, lam.data(), sizeof(double) * k, cudaMemcpyHostToDevice, s_);
  if (kind_ == BG_PRECOND_LEARNED)
    k_corrections<D, true><<<k, 256, 0, s_>>>(X_, HX_, rows_, diag_, lam_, Er_, norms_, rows_, kind_,
                                              static_cast<const __nv_bfloat16*>(op_->ctx->learned));
  else
    k_corrections<D, false><<<k, 256, 0, s_>>>(X_, HX_, rows_, diag_, lam_, Er_, norms_, rows_, kind_, nullptr);
  std::vector<double> n2(k);
  cudaMemcpyAsync(n2.data(), norms_, sizeof(double) * k, cudaMemcpyDeviceToHost, s_);
  if ((rc = sync("corrections"))) return rc;
  std::vector<int> map;
  std::vector<double> sc;
  for (int j = 0; j < k; ++j) {
    const double nrm = std::sqrt(n2[j]);
    if (!std::isfinite(nrm)) {
      err_ = "nonfinite reference correction";
      return BG_ENONFINITE;
    }
    if (nrm <= 32.0 * kEps) {
      stats_.dropped += 1;
      continue;
    }
    map.push_back(j);
    sc.push_back(1.0 / nrm);
  }
  *kept = (int)map.size();
  if (map.empty()) return BG_OK;
  cudaMemcpyAsync(map_, map.data(), sizeof(int) * map.size(), cudaMemcpyHostToDevice, s_);
  cudaMemcpyAsync(scale_, sc.data(), sizeof(double) * sc.size(), cudaMemcpyHostToDevice, s_);
  const dim3 grid((unsigned)std::min<int64_t>((rows_ + 255) / 256, 512), (unsigned)map.size());
  k_pick_scale<D><<<grid, 256, 0, s_>>>(Er_, rows_, map_, scale_, E_, rows_);
  if ((rc = sync("normalize"))) return rc;
  return check("corrections");
}

// Rank repair: rotate the basis to its Ritz vectors (S = I, H_r = diag lambda), project
// the raw corrections out of it twice, orthonormalise the block with the 1e-12 floor.
template <class T>
int Solver<T>::repair(int m, int* kept) {
  stats_.repairs += 1;
  int rc;
  std::vector<T> cm((size_t)m * m);
  for (int j = 0; j < m; ++j)
    for (int i = 0; i < m; ++i) cm[i + (size_t)j * m] = C_[i + (size_t)j * cap_];
  if ((rc = rotate(V_, m, cm.data(), m, X_))) return rc;
  if ((rc = rotate(HV_, m, cm.data(), m, HX_))) return rc;
  std::swap(V_, X_);
  std::swap(HV_, HX_);
  for (int j = 0; j < m; ++j)
    for (int i = 0; i < m; ++i) {
      const bool d = i == j;
      S_[i + (size_t)j * cap_] = T(d ? 1.0 : 0.0);
      L_[i + (size_t)j * cap_] = T(d ? 1.0 : 0.0);
      Hr_[i + (size_t)j * cap_] = T(d ? values_[i] : 0.0);
      C_[i + (size_t)j * cap_] = T(d ? 1.0 : 0.0);
    }
  int k = *kept;
  if (k == 0) return BG_OK;
  // two projections E <- E - V (V^H E)
  std::vector<T> P((size_t)m * k);
  for (int pass = 0; pass < 2; ++pass) {
    if ((rc = gram(V_, m, E_, k, P.data(), m))) return rc;
    for (auto& p : P) p = -p;
    if ((rc = rotate(V_, m, P.data(), k, E_, true))) return rc;
  }
  // in-block orthonormalisation: Gram G = E^H E, Cholesky-QR with the dependence floor
  std::vector<T> G((size_t)k * k), R((size_t)k * k, T(0));
  if ((rc = gram(E_, k, E_, k, G.data(), k))) return rc;
  std::vector<int> keep;
  std::vector<T> Q((size_t)k * k, T(0));  // coefficient of the orthonormal columns
  for (int j = 0; j < k; ++j) {
    // q = e_j - sum_{kept c} (q_c^H e_j) q_c, in coefficient space with metric G
    std::vector<T> q(k, T(0));
    q[j] = T(1);
    for (size_t c = 0; c < keep.size(); ++c) {
      const T* qc = Q.data() + c * k;
      T dot = T(0);  // q_c^H G e_j
      for (int a = 0; a < k; ++a) dot += dense::conj(qc[a]) * G[a + (size_t)j * k];
      for (int a = 0; a < k; ++a) q[a] -= dot * qc[a];
    }
    double nn = 0.0;  // q^H G q
    for (int a = 0; a < k; ++a)
      for (int b = 0; b < k; ++b) nn += dense::re(dense::conj(q[a]) * G[a + (size_t)b * k] * q[b]);
    const double len = std::sqrt(std::max(nn, 0.0));
    if (!(len > kDependence)) {
      stats_.dropped += 1;
      continue;
    }
    for (int a = 0; a < k; ++a) Q[keep.size() * k + a] = q[a] / len;
    keep.push_back(j);
  }
  const int kk = std::min<int>((int)keep.size(), cap_ - m);
  *kept = kk;
  if (kk == 0) return BG_OK;
  if ((rc = rotate(E_, k, Q.data(), kk, Er_))) return rc;
  std::swap(E_, Er_);
  return BG_OK;
}

template <class T>
int Solver<T>::contract(int m) {
  stats_.contractions += 1;
  std::vector<T> cn((size_t)m * n_);
  for (int j = 0; j < n_; ++j)
    for (int i = 0; i < m; ++i) cn[i + (size_t)j * m] = C_[i + (size_t)j * cap_];
  int rc = rotate(V_, m, cn.data(), n_, X_);
  if (!rc) rc = rotate(HV_, m, cn.data(), n_, HX_);
  if (rc) return rc;
  std::swap(V_, X_);
  std::swap(HV_, HX_);
  return refresh(n_);
}

template <class T>
int Solver<T>::run(const T* start, const double* diagonal, double* values_out, T* vectors_out, int32_t* converged,
                   bg_davidson_stats* st) {
  const size_t rc_ = (size_t)rows_ * cap_;
  int rc;
  if ((rc = alloc(&V_, rc_)) || (rc = alloc(&HV_, rc_)) || (rc = alloc(&X_, rc_)) || (rc = alloc(&HX_, rc_)) ||
      (rc = alloc(&E_, rc_)) || (rc = alloc(&Er_, rc_)) || (rc = alloc(&HE_, rc_)))
    return rc;
  part_elems_ = std::max<size_t>((size_t)cap_ * cap_ * 8, (size_t)8 * 148 * 32 * 32);
  if ((rc = alloc(&part_, part_elems_)) || (rc = alloc(&small_, (size_t)cap_ * cap_)) ||
      (rc = alloc(&coef_, (size_t)cap_ * cap_)) || (rc = alloc(&diag_, rows_)) || (rc = alloc(&lam_, cap_)) ||
      (rc = alloc(&norms_, cap_)) || (rc = alloc(&scale_, cap_)) || (rc = alloc(&map_, cap_)))
    return rc;
  S_.assign((size_t)cap_ * cap_, T(0));
  Hr_ = S_;
  L_ = S_;
  C_ = S_;
  cudaMemcpyAsync(V_, start, sizeof(T) * (size_t)rows_ * n_, cudaMemcpyHostToDevice, s_);
  cudaMemcpyAsync(diag_, diagonal, sizeof(double) * rows_, cudaMemcpyHostToDevice, s_);
  if ((rc = sync("upload"))) return rc;
  if ((rc = apply(V_, HV_, n_))) return rc;
  if ((rc = gram(V_, n_, V_, n_, S_.data(), cap_))) return rc;
  if (!dense::cholesky_extend(S_.data(), cap_, L_.data(), 0, n_)) {
    err_ = "reference Davidson start is numerically dependent";
    return BG_EINVAL;
  }
  if ((rc = gram(V_, n_, HV_, n_, Hr_.data(), cap_))) return rc;
  if ((rc = eigen(n_))) return rc;
  int m = n_;
  std::vector<int> active(n_);
  for (int i = 0; i < n_; ++i) active[i] = i;
  std::vector<char> conv(n_, 0);
  old_.assign(n_, 0.0);
  int iterations = 0;
  for (int step = 0; step < o_.max_iterations; ++step) {
    if (m + (int)active.size() > cap_ && m > n_) {
      if ((rc = contract(m))) return rc;
      m = n_;
    }
    if (m + (int)active.size() > cap_ && cap_ < rows_) {
      err_ = "capacity cannot hold the active correction block; use at least 2*bands";
      return BG_EINVAL;
    }
    int k = 0;
    if ((rc = corrections(active, m, diagonal, &k))) return rc;
    bool need_repair = (m + k > cap_) || k == 0;
    if (!need_repair) {
      cudaMemcpyAsync(V_ + (size_t)m * rows_, E_, sizeof(T) * (size_t)k * rows_, cudaMemcpyDeviceToDevice, s_);
      if ((rc = gram(V_, m + k, V_ + (size_t)m * rows_, k, S_.data() + (size_t)m * cap_, cap_))) return rc;
      for (int j = m; j < m + k; ++j)
        for (int i = 0; i <= j; ++i) S_[j + (size_t)i * cap_] = dense::conj(S_[i + (size_t)j * cap_]);
      if (!dense::cholesky_extend(S_.data(), cap_, L_.data(), m, m + k)) need_repair = true;
    }
    if (need_repair) {
      if ((rc = repair(m, &k))) return rc;
      if (k > 0) {
        cudaMemcpyAsync(V_ + (size_t)m * rows_, E_, sizeof(T) * (size_t)k * rows_, cudaMemcpyDeviceToDevice, s_);
        if ((rc = gram(V_, m + k, V_ + (size_t)m * rows_, k, S_.data() + (size_t)m * cap_, cap_))) return rc;
        for (int j = m; j < m + k; ++j)
          for (int i = 0; i <= j; ++i) S_[j + (size_t)i * cap_] = dense::conj(S_[i + (size_t)j * cap_]);
        if (!dense::cholesky_extend(S_.data(), cap_, L_.data(), m, m + k)) {
          err_ = "reference overlap remains dependent after repair";
          return BG_EINVAL;
        }
      }
    }
    for (int i = 0; i < n_; ++i) old_[i] = values_[i];
    if (k > 0) {
      if ((rc = apply(V_ + (size_t)m * rows_, HV_ + (size_t)m * rows_, k))) return rc;
      if ((rc = gram(V_, m + k, HV_ + (size_t)m * rows_, k, Hr_.data() + (size_t)m * cap_, cap_))) return rc;
      for (int j = m; j < m + k; ++j)
        for (int i = 0; i <= j; ++i) Hr_[j + (size_t)i * cap_] = dense::conj(Hr_[i + (size_t)j * cap_]);
      m += k;
      if ((rc = eigen(m))) return rc;
    } else if (need_repair) {
      // basis rotated to its Ritz vectors: C = I, values unchanged
    }
    active.clear();
    double dmax = 0.0;
    for (int i = 0; i < n_; ++i) {
      const double change = std::fabs(values_[i] - old_[i]);
      conv[i] = change < band_threshold(i);
      if (!conv[i]) active.push_back(i);
      dmax = std::max(dmax, change);
    }
    iterations = step + 1;
    if (kind_ == BG_PRECOND_LEARNED && !active.empty()) {
      // TPA fallback: the largest Ritz change has not fallen below its best for
      // kStallSteps iterations, or half the iteration budget is spent
      if (dmax < best_change_) {
        best_change_ = dmax;
        stalled_ = 0;
      } else {
        ++stalled_;
      }
      if (stalled_ >= kStallSteps || 2 * iterations >= o_.max_iterations) {
        kind_ = BG_PRECOND_TPA;
        stats_.fallbacks = 1;
      }
    }
    if (active.empty() || iterations == o_.max_iterations) break;
    if (m + (int)active.size() > cap_) {
      if ((rc = contract(m))) return rc;
      m = n_;
    }
  }
  // finish: X = V C[:, :n]
  std::vector<T> cn((size_t)m * n_);
  for (int j = 0; j < n_; ++j)
    for (int i = 0; i < m; ++i) cn[i + (size_t)j * m] = C_[i + (size_t)j * cap_];
  if ((rc = rotate(V_, m, cn.data(), n_, X_))) return rc;
  cudaMemcpyAsync(vectors_out, X_, sizeof(T) * (size_t)rows_ * n_, cudaMemcpyDeviceToHost, s_);
  if ((rc = sync("finish"))) return rc;
  for (int i = 0; i < n_; ++i) {
    values_out[i] = values_[i];
    converged[i] = conv[i] ? 1 : 0;
    stats_.converged_count += conv[i] ? 1 : 0;
  }
  stats_.iterations = iterations;
  if (st) *st = stats_;
  return BG_OK;
}

}  // namespace
}  // namespace bg

using namespace bg;

extern "C" int bg_davidson_solve(bg_op* op, const double* start, const double* diagonal,
                                 const bg_davidson_options* options, double* eigenvalues, double* eigenvectors,
                                 int32_t* converged, bg_davidson_stats* stats) {
  if (!op || !start || !diagonal || !options || !eigenvalues || !eigenvectors || !converged)
    return fail(op ? op->ctx : nullptr, BG_EINVAL, "null argument");
  const bg_davidson_options o = *options;
  const int64_t dim = op->rows;
  const int64_t n = o.bands;
  const int64_t cap = std::min<int64_t>(o.capacity == 0 ? 2 * n : o.capacity, dim);
  // crates/dft-solvers/src/ref_davidson.rs:133-146
  const bool bad = n == 0 || n > dim || cap < std::min<int64_t>(2 * n, dim) || o.occupied > n || o.occupied < 0 ||
                   o.max_iterations <= 0 || !std::isfinite(o.threshold) || o.threshold <= 0.0 || cap > op->cap ||
                   o.preconditioner < BG_PRECOND_SMOOTH || o.preconditioner > BG_PRECOND_LEARNED ||
                   (o.apply_precision != BG_PREC_FP64 && o.apply_precision != BG_PREC_FP32);
  if (bad) return fail(op->ctx, BG_EINVAL, "reference Davidson dimensions/threshold/start (capacity must also fit the operator)");
  if (o.preconditioner == BG_PRECOND_LEARNED && !op->ctx->learned)
    return fail(op->ctx, BG_EINVAL, "learned preconditioner requested but no network was set (bg_learned_set)");
  const size_t per = op->gamma ? 1 : 2;
  for (size_t i = 0; i < (size_t)dim * n * per; ++i)
    if (!std::isfinite(start[i])) return fail(op->ctx, BG_ENONFINITE, "reference Davidson start not finite");
  for (int64_t i = 0; i < dim; ++i)
    if (!std::isfinite(diagonal[i])) return fail(op->ctx, BG_ENONFINITE, "reference Davidson diagonal not finite");
  if (!op->has_epoch) return fail(op->ctx, BG_EEPOCH, "potential was never set");
  {
    const cudaError_t de = cudaSetDevice(op->ctx->device);
    if (de != cudaSuccess) return cuda_fail(op->ctx, de, "cudaSetDevice");
  }
  int rc;
  std::string err;
  if (per == 1) {
    Solver<double> s(op, (int)n, (int)cap, o);
    rc = s.run(start, diagonal, eigenvalues, eigenvectors, converged, stats);
    err = s.error();
  } else {
    Solver<std::complex<double>> s(op, (int)n, (int)cap, o);
    rc = s.run(reinterpret_cast<const std::complex<double>*>(start), diagonal, eigenvalues,
               reinterpret_cast<std::complex<double>*>(eigenvectors), converged, stats);
    err = s.error();
  }
  if (rc != BG_OK) return fail(op->ctx, rc, err.empty() ? "reference Davidson failed" : err);
  return BG_OK;
}

// ------------------------------------------------------------------ dense operators
namespace bg {
int dense_apply(bg_op* op, const double* x, double* y, int64_t cols) {
  const int64_t n = op->rows;
  const dim3 grid((unsigned)((n + 63) / 64), (unsigned)((cols + 31) / 32));
  if (op->gamma)
    k_gemm_nn<double><<<grid, 128, 0, op->stream>>>(op->dense, n, x, n, y, n, n, (int)cols, (int)n, 0);
  else
    k_gemm_nn<double2><<<grid, 128, 0, op->stream>>>(reinterpret_cast<const double2*>(op->dense), n,
                                                    reinterpret_cast<const double2*>(x), n,
                                                    reinterpret_cast<double2*>(y), n, n, (int)cols, (int)n, 0);
  op->launches += 1;
  return BG_OK;
}
}  // namespace bg

extern "C" int bg_op_create_dense(bg_ctx* ctx, int64_t rows, const double* h, int32_t is_complex, int64_t capacity,
                                  bg_op** out) {
  if (!ctx || !h || !out) return fail(ctx, BG_EINVAL, "null argument");
  if (rows < 1 || rows > (1 << 16) || capacity < 1 || capacity > 65535) return fail(ctx, BG_ESHAPE, "dense operator size");
  const size_t per = is_complex ? 2 : 1;
  const size_t count = (size_t)rows * rows * per;
  for (size_t i = 0; i < count; ++i)
    if (!std::isfinite(h[i])) return fail(ctx, BG_ENONFINITE, "dense operator not finite");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
  auto op = std::make_unique<bg_op>();
  op->ctx = ctx;
  op->is_dense = true;
  op->gamma = !is_complex;
  op->rows = rows;
  op->cap = capacity;
  op->cap_units = capacity;
  op->has_epoch = true;
  auto buf = std::make_unique<DevBuf>();
  buf->bytes = count * sizeof(double);
  if ((e = cudaMalloc(&buf->p, buf->bytes)) != cudaSuccess) return fail(ctx, BG_ENOMEM, "cudaMalloc");
  if ((e = cudaMemcpy(buf->p, h, buf->bytes, cudaMemcpyHostToDevice)) != cudaSuccess) return cuda_fail(ctx, e, "copy");
  op->dense = static_cast<double*>(buf->p);
  op->bufs.push_back(std::move(buf));
  auto stage = [&](DevBuf** keep) -> int {
    auto b = std::make_unique<DevBuf>();
    b->bytes = (size_t)rows * capacity * per * sizeof(double);
    if (cudaMalloc(&b->p, b->bytes) != cudaSuccess) return BG_ENOMEM;
    *keep = b.get();
    op->bufs.push_back(std::move(b));
    return BG_OK;
  };
  if (stage(&op->xs) || stage(&op->ys)) return fail(ctx, BG_ENOMEM, "cudaMalloc");
  op->diag.resize(rows);
  for (int64_t i = 0; i < rows; ++i) op->diag[i] = h[(i + (size_t)i * rows) * per];
  if ((e = cudaMallocHost(&op->err_host, sizeof(int) * 4)) != cudaSuccess) return cuda_fail(ctx, e, "cudaMallocHost");
  void* errp = nullptr;
  if ((e = cudaMalloc(&errp, sizeof(int) * 4)) != cudaSuccess) return fail(ctx, BG_ENOMEM, "cudaMalloc");
  auto eb = std::make_unique<DevBuf>();
  eb->p = errp;
  eb->bytes = sizeof(int) * 4;
  op->bufs.push_back(std::move(eb));
  op->t.err = static_cast<int*>(errp);
  cudaMemset(op->t.err, 0, sizeof(int) * 4);
  if ((e = cudaStreamCreateWithFlags(&op->stream, cudaStreamNonBlocking)) != cudaSuccess)
    return cuda_fail(ctx, e, "cudaStreamCreate");
  op->own_stream = true;
  *out = op.release();
  return BG_OK;
}
