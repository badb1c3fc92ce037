// Oracle (test infrastructure only): CPU FP64 restatement of the reference's
// Hamiltonian apply H.x for one k point (complex coefficients) and for the real
// Gamma ORC rows (two real columns per complex FFT).  Only tests/, the smoke check
// and bench.py's cpu_baseline leg load this library; the product never links it.
//
// Follows (paths inside the reference project):
//   complex apply  crates/dft-physics/src/distributed_complex.rs:340-386
//                  (out = local(x) + T.x + P (D (P^H x)); coupling loop :326-336)
//   Gamma apply    crates/dft-physics/src/distributed_real_gamma.rs:1062-1264
//                  (pair pack :654-689, unpack even/odd :1307-1341, kinetic
//                  :1343-1347, P^T x :957-1017, coupling :1184-1195, P W :1200-1248)
//   local part     crates/dft-solvers/src/distributed_fft.rs:1198-1288
//                  (scatter, pruned inverse 3D FFT without scale, x V(r), forward
//                  3D FFT, x 1/N, gather; conventions docs/physics-conventions.md:61-78)
//   diagonal       crates/dft-physics/src/distributed_complex.rs:29-53
//
// The 1D transforms are a self-contained mixed-radix Stockham FFT (twiddles in long
// double).  Pruning follows the reference's stick plan: the first axis is
// transformed only on occupied sticks, the middle axis only on planes of the last
// axis that hold coefficients, and the last axis on every line.
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <omp.h>

using cd = std::complex<double>;

namespace {

struct Plan1D {
  int n = 0;
  std::vector<int> radices;
  std::vector<cd> tw_inv, tw_fwd;  // exp(+-2 pi i q / n)
};

Plan1D make_plan(int n) {
  Plan1D p;
  p.n = n;
  int m = n;
  for (int r : {4, 2, 3, 5}) {
    while (m % r == 0) {
      p.radices.push_back(r);
      m /= r;
    }
  }
  if (m != 1) p.radices.push_back(m);  // generic prime factor (direct DFT)
  p.tw_inv.resize(n);
  p.tw_fwd.resize(n);
  const long double two_pi = 6.283185307179586476925286766559005768L;
  for (int q = 0; q < n; ++q) {
    long double a = two_pi * (long double)q / (long double)n;
    double c = (double)cosl(a), s = (double)sinl(a);
    p.tw_inv[q] = cd(c, s);
    p.tw_fwd[q] = cd(c, -s);
  }
  return p;
}

// Stockham autosort, out-of-place ping-pong; `sign` +1 inverse, -1 forward.
void fft_line(const Plan1D& p, cd* data, int stride, cd* a, cd* b, int sign) {
  const int n = p.n;
  const std::vector<cd>& tw = sign > 0 ? p.tw_inv : p.tw_fwd;
  for (int i = 0; i < n; ++i) a[i] = data[(size_t)i * stride];
  int ns = 1;
  cd v[64];
  for (int r : p.radices) {
    const int span = n / r;
    for (int j = 0; j < span; ++j) {
      const int k = j % ns;
      const int step = n / (ns * r);
      for (int t = 0; t < r; ++t) v[t] = a[j + t * span] * tw[(t * k * step) % n];
      const int base = (j / ns) * ns * r + k;
      for (int u = 0; u < r; ++u) {
        cd acc = 0.0;
        for (int t = 0; t < r; ++t) acc += v[t] * tw[((t * u) % r) * (n / r)];
        b[base + u * ns] = acc;
      }
    }
    std::swap(a, b);
    ns *= r;
  }
  for (int i = 0; i < n; ++i) data[(size_t)i * stride] = a[i];
}

struct LocalPlan {
  int n0, n1, n2;
  Plan1D p0, p1, p2;
  std::vector<int64_t> index;            // flat C-order FFT index of every row
  std::vector<int> sticks;               // occupied (j,k) of axis-0 lines: j*n2+k
  std::vector<int> planes;               // occupied k values (last axis)
};

LocalPlan make_local(int n0, int n1, int n2, int64_t npw, const int64_t* index) {
  LocalPlan L;
  L.n0 = n0; L.n1 = n1; L.n2 = n2;
  L.p0 = make_plan(n0); L.p1 = make_plan(n1); L.p2 = make_plan(n2);
  L.index.assign(index, index + npw);
  std::vector<char> st((size_t)n1 * n2, 0), pl(n2, 0);
  for (int64_t g = 0; g < npw; ++g) {
    int64_t f = index[g];
    int k = (int)(f % n2);
    int j = (int)((f / n2) % n1);
    st[(size_t)j * n2 + k] = 1;
    pl[k] = 1;
  }
  for (int s = 0; s < n1 * n2; ++s) if (st[s]) L.sticks.push_back(s);
  for (int k = 0; k < n2; ++k) if (pl[k]) L.planes.push_back(k);
  return L;
}

// h = gather( FFT_fwd( V * IFFT(scatter(c)) ) ) / N, for one complex vector.
void local_apply(const LocalPlan& L, const double* v, const cd* c, cd* h, std::vector<cd>& box,
                 std::vector<cd>& sa, std::vector<cd>& sb) {
  const int n0 = L.n0, n1 = L.n1, n2 = L.n2;
  const size_t N = (size_t)n0 * n1 * n2;
  box.assign(N, cd(0.0, 0.0));
  const int64_t npw = (int64_t)L.index.size();
  for (int64_t g = 0; g < npw; ++g) box[L.index[g]] = c[g];
  // inverse: axis 0 on occupied sticks, axis 1 on occupied last-axis planes, axis 2 everywhere
  for (int s : L.sticks) fft_line(L.p0, box.data() + s, n1 * n2, sa.data(), sb.data(), +1);
  for (int i = 0; i < n0; ++i)
    for (int k : L.planes) fft_line(L.p1, box.data() + (size_t)i * n1 * n2 + k, n2, sa.data(), sb.data(), +1);
  for (size_t line = 0; line < (size_t)n0 * n1; ++line)
    fft_line(L.p2, box.data() + line * n2, 1, sa.data(), sb.data(), +1);
  for (size_t f = 0; f < N; ++f) box[f] *= v[f];
  for (size_t line = 0; line < (size_t)n0 * n1; ++line)
    fft_line(L.p2, box.data() + line * n2, 1, sa.data(), sb.data(), -1);
  for (int i = 0; i < n0; ++i)
    for (int k : L.planes) fft_line(L.p1, box.data() + (size_t)i * n1 * n2 + k, n2, sa.data(), sb.data(), -1);
  for (int s : L.sticks) fft_line(L.p0, box.data() + s, n1 * n2, sa.data(), sb.data(), -1);
  const double inv_n = 1.0 / (double)N;
  for (int64_t g = 0; g < npw; ++g) h[g] = box[L.index[g]] * inv_n;
}

int max_len(const LocalPlan& L) { return std::max(L.n0, std::max(L.n1, L.n2)); }

}  // namespace

extern "C" {

// Complex (k point) apply.  Layouts: x, y, proj are column-major complex with
// interleaved (re, im) doubles; index = flat C-order FFT index per row; v is the
// full real grid in C order; couplings concatenated per atom (count*count,
// row-major).  Returns 0, or 1 on a shape error.
int oracle_apply_complex(int n0, int n1, int n2, int64_t npw, const int64_t* index, const double* v,
                         const double* kinetic, int nproj, const double* proj, int natoms,
                         const int* channels, const double* couplings, const double* x, double* y,
                         int m, int threads) {
  if (n0 <= 0 || n1 <= 0 || n2 <= 0 || npw <= 0 || m < 0) return 1;
  LocalPlan L = make_local(n0, n1, n2, npw, index);
  const cd* X = reinterpret_cast<const cd*>(x);
  cd* Y = reinterpret_cast<cd*>(y);
  const cd* P = reinterpret_cast<const cd*>(proj);
  if (threads > 0) omp_set_num_threads(threads);
  // Local part + kinetic, one column per task.
#pragma omp parallel
  {
    std::vector<cd> box, sa(max_len(L)), sb(max_len(L));
#pragma omp for schedule(dynamic)
    for (int c = 0; c < m; ++c) {
      local_apply(L, v, X + (size_t)c * npw, Y + (size_t)c * npw, box, sa, sb);
      for (int64_t g = 0; g < npw; ++g) Y[(size_t)c * npw + g] += kinetic[g] * X[(size_t)c * npw + g];
    }
  }
  if (nproj == 0) return 0;
  // W = P^H X (nproj x m), then D per atom, then Y += P W'.
  std::vector<cd> W((size_t)nproj * m), Wd((size_t)nproj * m);
#pragma omp parallel for collapse(2) schedule(static)
  for (int c = 0; c < m; ++c)
    for (int p = 0; p < nproj; ++p) {
      cd acc = 0.0;
      const cd* pc = P + (size_t)p * npw;
      const cd* xc = X + (size_t)c * npw;
      for (int64_t g = 0; g < npw; ++g) acc += std::conj(pc[g]) * xc[g];
      W[(size_t)c * nproj + p] = acc;
    }
  for (int c = 0; c < m; ++c) {
    int off = 0, coff = 0;
    for (int a = 0; a < natoms; ++a) {
      const int cnt = channels[a];
      for (int i = 0; i < cnt; ++i) {
        cd acc = 0.0;
        for (int j = 0; j < cnt; ++j) acc += couplings[coff + i * cnt + j] * W[(size_t)c * nproj + off + j];
        Wd[(size_t)c * nproj + off + i] = acc;
      }
      off += cnt;
      coff += cnt * cnt;
    }
  }
#pragma omp parallel for schedule(static)
  for (int c = 0; c < m; ++c) {
    cd* yc = Y + (size_t)c * npw;
    for (int p = 0; p < nproj; ++p) {
      const cd w = Wd[(size_t)c * nproj + p];
      const cd* pc = P + (size_t)p * npw;
      for (int64_t g = 0; g < npw; ++g) yc[g] += pc[g] * w;
    }
  }
  return 0;
}

// Real Gamma apply on ORC rows.  plus/minus: nh representative indices into the
// full sphere (plus[0] = minus[0] = 0); index: flat FFT index of every full-sphere
// position; kinetic: ORC-order kinetic (n rows); proj: real ORC projectors,
// column-major n x nproj; x, y: column-major n x m.
int oracle_apply_gamma(int n0, int n1, int n2, int64_t n, const int64_t* index, int64_t nh,
                       const int64_t* plus, const int64_t* minus, const double* v,
                       const double* kinetic, int nproj, const double* proj, int natoms,
                       const int* channels, const double* couplings, const double* x, double* y,
                       int m, int threads) {
  if (n0 <= 0 || n1 <= 0 || n2 <= 0 || n <= 0 || 2 * nh - 1 != n || m < 0) return 1;
  LocalPlan L = make_local(n0, n1, n2, n, index);
  const int pairs = (m + 1) / 2;
  const double r2 = std::sqrt(2.0);
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel
  {
    std::vector<cd> box, sa(max_len(L)), sb(max_len(L)), phi(n), h(n);
#pragma omp for schedule(dynamic)
    for (int t = 0; t < pairs; ++t) {
      const int ca = 2 * t;
      const bool hasb = 2 * t + 1 < m;
      const double* xa = x + (size_t)ca * n;
      const double* xb = hasb ? x + (size_t)(ca + 1) * n : nullptr;
      // pack (distributed_real_gamma.rs:654-689)
      phi[0] = cd(xa[0], hasb ? xb[0] : 0.0);
      for (int64_t i = 1; i < nh; ++i) {
        cd a = cd(xa[2 * i - 1], xa[2 * i]) / r2;
        cd b = hasb ? cd(xb[2 * i - 1], xb[2 * i]) / r2 : cd(0.0, 0.0);
        phi[plus[i]] = a + cd(-b.imag(), b.real());
        phi[minus[i]] = std::conj(a) + cd(b.imag(), b.real());
      }
      local_apply(L, v, phi.data(), h.data(), box, sa, sb);
      // unpack (distributed_real_gamma.rs:1307-1341)
      double* ya = y + (size_t)ca * n;
      double* yb = hasb ? y + (size_t)(ca + 1) * n : nullptr;
      ya[0] = h[0].real();
      if (hasb) yb[0] = h[0].imag();
      for (int64_t i = 1; i < nh; ++i) {
        cd hp = h[plus[i]], hm = h[minus[i]];
        cd even = (hp + std::conj(hm)) * 0.5;
        cd odd = (hp - std::conj(hm)) * 0.5;
        ya[2 * i - 1] = even.real() * r2;
        ya[2 * i] = even.imag() * r2;
        if (hasb) {
          yb[2 * i - 1] = odd.imag() * r2;
          yb[2 * i] = -odd.real() * r2;
        }
      }
      // kinetic (distributed_real_gamma.rs:1343-1347)
      for (int64_t j = 0; j < n; ++j) ya[j] += kinetic[j] * xa[j];
      if (hasb)
        for (int64_t j = 0; j < n; ++j) yb[j] += kinetic[j] * xb[j];
    }
  }
  if (nproj == 0) return 0;
  std::vector<double> Q((size_t)nproj * m), Wt((size_t)nproj * m);
#pragma omp parallel for collapse(2) schedule(static)
  for (int c = 0; c < m; ++c)
    for (int p = 0; p < nproj; ++p) {
      double acc = 0.0;
      const double* pc = proj + (size_t)p * n;
      const double* xc = x + (size_t)c * n;
      for (int64_t g = 0; g < n; ++g) acc += pc[g] * xc[g];
      Q[(size_t)c * nproj + p] = acc;
    }
  // coupling (distributed_real_gamma.rs:1184-1195): atom, band, j, k order
  int off = 0, coff = 0;
  for (int a = 0; a < natoms; ++a) {
    const int cnt = channels[a];
    for (int c = 0; c < m; ++c)
      for (int j = 0; j < cnt; ++j) {
        double val = 0.0;
        for (int k = 0; k < cnt; ++k) val += couplings[coff + j * cnt + k] * Q[(size_t)c * nproj + off + k];
        Wt[(size_t)c * nproj + off + j] = val;
      }
    off += cnt;
    coff += cnt * cnt;
  }
#pragma omp parallel for schedule(static)
  for (int c = 0; c < m; ++c) {
    double* yc = y + (size_t)c * n;
    for (int p = 0; p < nproj; ++p) {
      const double w = Wt[(size_t)c * nproj + p];
      const double* pc = proj + (size_t)p * n;
      for (int64_t g = 0; g < n; ++g) yc[g] += pc[g] * w;
    }
  }
  return 0;
}

// Complex 3D transforms of a full grid (oracle of the FFT conventions):
// sign +1: f(r) = sum_G f(G) e^{+iGr} (no scale); sign -1: f(G) = (1/N) sum_r f(r) e^{-iGr}.
int oracle_fft3d(int n0, int n1, int n2, double* data, int sign) {
  if (n0 <= 0 || n1 <= 0 || n2 <= 0 || (sign != 1 && sign != -1)) return 1;
  Plan1D p0 = make_plan(n0), p1 = make_plan(n1), p2 = make_plan(n2);
  cd* box = reinterpret_cast<cd*>(data);
  int mx = std::max(n0, std::max(n1, n2));
  std::vector<cd> sa(mx), sb(mx);
  for (int j = 0; j < n1 * n2; ++j) fft_line(p0, box + j, n1 * n2, sa.data(), sb.data(), sign);
  for (int i = 0; i < n0; ++i)
    for (int k = 0; k < n2; ++k) fft_line(p1, box + (size_t)i * n1 * n2 + k, n2, sa.data(), sb.data(), sign);
  for (int line = 0; line < n0 * n1; ++line) fft_line(p2, box + (size_t)line * n2, 1, sa.data(), sb.data(), sign);
  if (sign < 0) {
    const double s = 1.0 / ((double)n0 * n1 * n2);
    for (size_t f = 0; f < (size_t)n0 * n1 * n2; ++f) box[f] *= s;
  }
  return 0;
}

}  // extern "C"
