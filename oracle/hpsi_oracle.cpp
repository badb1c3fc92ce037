// Oracle (test infrastructure only): CPU FP64 restatement of the reference's
// Hamiltonian apply H.x for one k point (complex coefficients) and for the real
// Gamma ORC rows (two real columns per complex FFT).  Only tests/, the smoke check
// and bench.py's cpu_baseline leg and reference arm load this library; the product
// never links it.
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
// The 1D transforms are a self-contained mixed-radix Stockham FFT (twiddles per stage,
// computed in long double; radix-2/3/4/5 butterflies written out, other primes as a
// direct DFT), run on four lines at once with the lines in the fastest index so the
// butterflies vectorise (the reference runs rustfft's SIMD lanes over batches of lines,
// distributed_fft.rs:208-221).  Pruning follows the reference's stick plan: lines of
// the first transformed axis only where coefficients sit, the middle axis only on the
// planes that hold them, the last axis everywhere.  On the C-order box [i][j][k] the
// sticks are the contiguous k lines at occupied (i, j), the planes the occupied i.
//
// The nonlocal part (P^H x, D, P W) is three dense products; oracle.py forms them
// with numpy's BLAS, as the reference forms them with faer/MKL GEMMs.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>

using cd = std::complex<double>;

namespace {

constexpr int LB = 4;  // lines per batch (the fastest index of a batch buffer)

struct Stage {
  int r = 0, ns = 0, span = 0;
  std::vector<double> wr, wi;  // twiddle (k, t) at [k * (r - 1) + t - 1]: exp(+2 pi i t k / (ns r))
};

struct Plan1D {
  int n = 0;
  std::vector<Stage> st;
};

Plan1D make_plan(int n) {
  Plan1D p;
  p.n = n;
  std::vector<int> radices;
  int m = n;
  for (int r : {4, 2, 3, 5}) {
    while (m % r == 0) {
      radices.push_back(r);
      m /= r;
    }
  }
  for (int f = 7; m > 1; f += 2) {
    while (m % f == 0) {
      radices.push_back(f);
      m /= f;
    }
  }
  const long double two_pi = 6.283185307179586476925286766559005768L;
  int ns = 1;
  for (int r : radices) {
    Stage s;
    s.r = r;
    s.ns = ns;
    s.span = n / r;
    s.wr.resize((size_t)ns * (r - 1));
    s.wi.resize((size_t)ns * (r - 1));
    for (int k = 0; k < ns; ++k)
      for (int t = 1; t < r; ++t) {
        const long double a = two_pi * (long double)(t * k) / (long double)(ns * r);
        s.wr[(size_t)k * (r - 1) + t - 1] = (double)cosl(a);
        s.wi[(size_t)k * (r - 1) + t - 1] = (double)sinl(a);
      }
    p.st.push_back(std::move(s));
    ns *= r;
  }
  return p;
}

// Four doubles as one value (GCC vector extension; one AVX2 register).
typedef double vd __attribute__((vector_size(32), aligned(8)));
inline vd ldv(const double* p) {
  vd v;
  std::memcpy(&v, p, sizeof(vd));
  return v;
}
inline void stv(double* p, const vd& v) { std::memcpy(p, &v, sizeof(vd)); }

// A batch: element e of line l at re[e * LB + l], im[e * LB + l].  One Stockham stage of
// radix R from (ar, ai) to (br, bi) with kernel exp(sign 2 pi i t u / R): the R inputs of
// butterfly j sit `span` elements apart and are twiddled by exp(sign 2 pi i t k / (ns R)).
template <int R>
void stage_r(const Stage& S, const double* __restrict__ ar, const double* __restrict__ ai, double* __restrict__ br,
             double* __restrict__ bi, int sign) {
  const int ns = S.ns, span = S.span;
  const double sg = (double)sign;
  int k = 0, jb = 0;
  for (int j = 0; j < span; ++j) {
    const int base = jb * ns * R + k;
    vd xr[R], xi[R];
    xr[0] = ldv(ar + (size_t)j * LB);
    xi[0] = ldv(ai + (size_t)j * LB);
    for (int t = 1; t < R; ++t) {
      const double c = S.wr[(size_t)k * (R - 1) + t - 1], s = sg * S.wi[(size_t)k * (R - 1) + t - 1];
      const vd a = ldv(ar + (size_t)(j + t * span) * LB), b = ldv(ai + (size_t)(j + t * span) * LB);
      xr[t] = a * c - b * s;
      xi[t] = a * s + b * c;
    }
    vd yr[R], yi[R];
    if constexpr (R == 2) {
      yr[0] = xr[0] + xr[1];
      yi[0] = xi[0] + xi[1];
      yr[1] = xr[0] - xr[1];
      yi[1] = xi[0] - xi[1];
    } else if constexpr (R == 4) {
      const vd s0r = xr[0] + xr[2], s0i = xi[0] + xi[2];
      const vd d0r = xr[0] - xr[2], d0i = xi[0] - xi[2];
      const vd s1r = xr[1] + xr[3], s1i = xi[1] + xi[3];
      const vd d1r = xr[1] - xr[3], d1i = xi[1] - xi[3];
      const vd er = -sg * d1i, ei = sg * d1r;  // sign i (x1 - x3)
      yr[0] = s0r + s1r;
      yi[0] = s0i + s1i;
      yr[2] = s0r - s1r;
      yi[2] = s0i - s1i;
      yr[1] = d0r + er;
      yi[1] = d0i + ei;
      yr[3] = d0r - er;
      yi[3] = d0i - ei;
    } else if constexpr (R == 3) {
      const double c = -0.5, sn = sg * 0.86602540378443864676372317075294;
      const vd t1r = xr[1] + xr[2], t1i = xi[1] + xi[2];
      const vd t2r = xr[0] + c * t1r, t2i = xi[0] + c * t1i;
      const vd t3r = sn * (xr[1] - xr[2]), t3i = sn * (xi[1] - xi[2]);
      yr[0] = xr[0] + t1r;
      yi[0] = xi[0] + t1i;
      yr[1] = t2r - t3i;
      yi[1] = t2i + t3r;
      yr[2] = t2r + t3i;
      yi[2] = t2i - t3r;
    } else if constexpr (R == 5) {
      const double c1 = 0.30901699437494742410229341718282, c2 = -0.80901699437494742410229341718282;
      const double s1 = sg * 0.95105651629515357211643933337938, s2 = sg * 0.58778525229247312916870595463907;
      const vd t1r = xr[1] + xr[4], t1i = xi[1] + xi[4];
      const vd t2r = xr[2] + xr[3], t2i = xi[2] + xi[3];
      const vd t3r = xr[1] - xr[4], t3i = xi[1] - xi[4];
      const vd t4r = xr[2] - xr[3], t4i = xi[2] - xi[3];
      const vd a1r = xr[0] + c1 * t1r + c2 * t2r, a1i = xi[0] + c1 * t1i + c2 * t2i;
      const vd a2r = xr[0] + c2 * t1r + c1 * t2r, a2i = xi[0] + c2 * t1i + c1 * t2i;
      const vd b1r = s1 * t3r + s2 * t4r, b1i = s1 * t3i + s2 * t4i;
      const vd b2r = s2 * t3r - s1 * t4r, b2i = s2 * t3i - s1 * t4i;
      yr[0] = xr[0] + t1r + t2r;
      yi[0] = xi[0] + t1i + t2i;
      yr[1] = a1r - b1i;
      yi[1] = a1i + b1r;
      yr[4] = a1r + b1i;
      yi[4] = a1i - b1r;
      yr[2] = a2r - b2i;
      yi[2] = a2i + b2r;
      yr[3] = a2r + b2i;
      yi[3] = a2i - b2r;
    }
    for (int u = 0; u < R; ++u) {
      stv(br + (size_t)(base + u * ns) * LB, yr[u]);
      stv(bi + (size_t)(base + u * ns) * LB, yi[u]);
    }
    if (++k == ns) {
      k = 0;
      ++jb;
    }
  }
}

// Other primes: a direct DFT with the length-r roots.
void stage_generic(const Stage& S, const double* ar, const double* ai, double* br, double* bi, int sign) {
  const int r = S.r, ns = S.ns, span = S.span;
  const long double two_pi = 6.283185307179586476925286766559005768L;
  std::vector<double> xr((size_t)r * LB), xi((size_t)r * LB);
  for (int j = 0; j < span; ++j) {
    const int k = j % ns, base = (j / ns) * ns * r + k;
    for (int t = 0; t < r; ++t) {
      const double c = t ? S.wr[(size_t)k * (r - 1) + t - 1] : 1.0;
      const double s = t ? sign * S.wi[(size_t)k * (r - 1) + t - 1] : 0.0;
      for (int l = 0; l < LB; ++l) {
        const double a = ar[(size_t)(j + t * span) * LB + l], b = ai[(size_t)(j + t * span) * LB + l];
        xr[(size_t)t * LB + l] = a * c - b * s;
        xi[(size_t)t * LB + l] = a * s + b * c;
      }
    }
    for (int u = 0; u < r; ++u)
      for (int l = 0; l < LB; ++l) {
        double accr = xr[l], acci = xi[l];
        for (int t = 1; t < r; ++t) {
          const long double a = two_pi * (long double)((t * u) % r) / (long double)r;
          const double c = (double)cosl(a), s = sign * (double)sinl(a);
          accr += xr[(size_t)t * LB + l] * c - xi[(size_t)t * LB + l] * s;
          acci += xr[(size_t)t * LB + l] * s + xi[(size_t)t * LB + l] * c;
        }
        br[(size_t)(base + u * ns) * LB + l] = accr;
        bi[(size_t)(base + u * ns) * LB + l] = acci;
      }
  }
}

void stage(const Stage& S, const double* ar, const double* ai, double* br, double* bi, int sign) {
  switch (S.r) {
    case 2: stage_r<2>(S, ar, ai, br, bi, sign); break;
    case 3: stage_r<3>(S, ar, ai, br, bi, sign); break;
    case 4: stage_r<4>(S, ar, ai, br, bi, sign); break;
    case 5: stage_r<5>(S, ar, ai, br, bi, sign); break;
    default: stage_generic(S, ar, ai, br, bi, sign); break;
  }
}

// Transform the batch in (re, im) in place (scratch (tr, ti) of the same size).
void fft_batch(const Plan1D& p, double* re, double* im, double* tr, double* ti, int sign) {
  double *ar = re, *ai = im, *br = tr, *bi = ti;
  for (const Stage& S : p.st) {
    stage(S, ar, ai, br, bi, sign);
    std::swap(ar, br);
    std::swap(ai, bi);
  }
  if (ar != re) {
    std::memcpy(re, ar, sizeof(double) * p.n * LB);
    std::memcpy(im, ai, sizeof(double) * p.n * LB);
  }
}

struct Scratch {
  std::vector<double> re, im, tr, ti;
  explicit Scratch(int n) : re((size_t)n * LB), im((size_t)n * LB), tr((size_t)n * LB), ti((size_t)n * LB) {}
};

// Lines of length p.n starting at box + start[l] with element stride `stride`, in batches of LB.
void fft_lines(const Plan1D& p, cd* box, const size_t* start, int count, size_t stride, Scratch& s, int sign) {
  const int n = p.n;
  double* re = s.re.data();
  double* im = s.im.data();
  for (int l0 = 0; l0 < count; l0 += LB) {
    const int c = std::min(LB, count - l0);
    double* line[LB];
    for (int l = 0; l < LB; ++l) line[l] = reinterpret_cast<double*>(box + start[l0 + (l < c ? l : 0)]);
    const size_t st2 = 2 * stride;
    for (int e = 0; e < n; ++e)
      for (int l = 0; l < LB; ++l) {
        const double* q = line[l] + (size_t)e * st2;
        re[(size_t)e * LB + l] = q[0];
        im[(size_t)e * LB + l] = q[1];
      }
    fft_batch(p, re, im, s.tr.data(), s.ti.data(), sign);
    for (int e = 0; e < n; ++e)
      for (int l = 0; l < c; ++l) {
        double* q = line[l] + (size_t)e * st2;
        q[0] = re[(size_t)e * LB + l];
        q[1] = im[(size_t)e * LB + l];
      }
  }
}

struct LocalPlan {
  int n0, n1, n2;
  Plan1D p0, p1, p2;
  std::vector<int64_t> index;      // flat C-order FFT index of every row
  std::vector<size_t> sticks;      // starts of the k lines at occupied (i, j)
  std::vector<size_t> ylines;      // starts of the j lines (stride n2) in occupied planes i
  std::vector<size_t> xlines;      // starts of every i line (stride n1 n2)
};

LocalPlan make_local(int n0, int n1, int n2, int64_t npw, const int64_t* index) {
  LocalPlan L;
  L.n0 = n0;
  L.n1 = n1;
  L.n2 = n2;
  L.p0 = make_plan(n0);
  L.p1 = make_plan(n1);
  L.p2 = make_plan(n2);
  L.index.assign(index, index + npw);
  std::vector<char> st((size_t)n0 * n1, 0), pl(n0, 0);
  for (int64_t g = 0; g < npw; ++g) {
    const int64_t f = index[g];
    const int64_t ij = f / n2;
    st[(size_t)ij] = 1;
    pl[(size_t)(ij / n1)] = 1;
  }
  for (size_t ij = 0; ij < (size_t)n0 * n1; ++ij)
    if (st[ij]) L.sticks.push_back(ij * n2);
  for (int i = 0; i < n0; ++i)
    if (pl[i])
      for (int k = 0; k < n2; ++k) L.ylines.push_back((size_t)i * n1 * n2 + k);
  for (size_t jk = 0; jk < (size_t)n1 * n2; ++jk) L.xlines.push_back(jk);
  return L;
}

// h = gather( FFT_fwd( V * IFFT(scatter(c)) ) ) / N, for one complex vector.
void local_apply(const LocalPlan& L, const double* v, const cd* c, cd* h, std::vector<cd>& box, Scratch& s) {
  const int n0 = L.n0, n1 = L.n1, n2 = L.n2;
  const size_t N = (size_t)n0 * n1 * n2;
  box.assign(N, cd(0.0, 0.0));
  const int64_t npw = (int64_t)L.index.size();
  for (int64_t g = 0; g < npw; ++g) box[L.index[g]] = c[g];
  fft_lines(L.p2, box.data(), L.sticks.data(), (int)L.sticks.size(), 1, s, +1);
  fft_lines(L.p1, box.data(), L.ylines.data(), (int)L.ylines.size(), (size_t)n2, s, +1);
  fft_lines(L.p0, box.data(), L.xlines.data(), (int)L.xlines.size(), (size_t)n1 * n2, s, +1);
  for (size_t f = 0; f < N; ++f) box[f] *= v[f];
  fft_lines(L.p0, box.data(), L.xlines.data(), (int)L.xlines.size(), (size_t)n1 * n2, s, -1);
  fft_lines(L.p1, box.data(), L.ylines.data(), (int)L.ylines.size(), (size_t)n2, s, -1);
  fft_lines(L.p2, box.data(), L.sticks.data(), (int)L.sticks.size(), 1, s, -1);
  const double inv_n = 1.0 / (double)N;
  for (int64_t g = 0; g < npw; ++g) h[g] = box[L.index[g]] * inv_n;
}

int max_len(const LocalPlan& L) { return std::max(L.n0, std::max(L.n1, L.n2)); }

}  // namespace

extern "C" {

// Local part plus kinetic of the complex (k point) apply.  Layouts: x, y column-major
// complex with interleaved (re, im) doubles; index = flat C-order FFT index per row;
// v is the full real grid in C order.  Returns 0, or 1 on a shape error.
int oracle_local_complex(int n0, int n1, int n2, int64_t npw, const int64_t* index, const double* v,
                         const double* kinetic, const double* x, double* y, int m, int threads) {
  if (n0 <= 0 || n1 <= 0 || n2 <= 0 || npw <= 0 || m < 0) return 1;
  LocalPlan L = make_local(n0, n1, n2, npw, index);
  const cd* X = reinterpret_cast<const cd*>(x);
  cd* Y = reinterpret_cast<cd*>(y);
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel
  {
    std::vector<cd> box;
    Scratch s(max_len(L));
#pragma omp for schedule(dynamic)
    for (int c = 0; c < m; ++c) {
      local_apply(L, v, X + (size_t)c * npw, Y + (size_t)c * npw, box, s);
      for (int64_t g = 0; g < npw; ++g) Y[(size_t)c * npw + g] += kinetic[g] * X[(size_t)c * npw + g];
    }
  }
  return 0;
}

// Local part plus kinetic of the real Gamma apply on ORC rows.  plus/minus: nh
// representative indices into the full sphere (plus[0] = minus[0] = 0); index: flat FFT
// index of every full-sphere position; kinetic: ORC-order kinetic (n rows); x, y:
// column-major n x m.
int oracle_local_gamma(int n0, int n1, int n2, int64_t n, const int64_t* index, int64_t nh, const int64_t* plus,
                       const int64_t* minus, const double* v, const double* kinetic, const double* x, double* y,
                       int m, int threads) {
  if (n0 <= 0 || n1 <= 0 || n2 <= 0 || n <= 0 || 2 * nh - 1 != n || m < 0) return 1;
  LocalPlan L = make_local(n0, n1, n2, n, index);
  const int pairs = (m + 1) / 2;
  const double r2 = std::sqrt(2.0);
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel
  {
    std::vector<cd> box, phi(n), h(n);
    Scratch s(max_len(L));
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
      local_apply(L, v, phi.data(), h.data(), box, s);
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
  return 0;
}

// Complex 3D transforms of a full grid (oracle of the FFT conventions):
// sign +1: f(r) = sum_G f(G) e^{+iGr} (no scale); sign -1: f(G) = (1/N) sum_r f(r) e^{-iGr}.
int oracle_fft3d(int n0, int n1, int n2, double* data, int sign) {
  if (n0 <= 0 || n1 <= 0 || n2 <= 0 || (sign != 1 && sign != -1)) return 1;
  Plan1D p0 = make_plan(n0), p1 = make_plan(n1), p2 = make_plan(n2);
  cd* box = reinterpret_cast<cd*>(data);
  Scratch s(std::max(n0, std::max(n1, n2)));
  std::vector<size_t> l0, l1, l2;
  for (size_t jk = 0; jk < (size_t)n1 * n2; ++jk) l0.push_back(jk);
  for (int i = 0; i < n0; ++i)
    for (int k = 0; k < n2; ++k) l1.push_back((size_t)i * n1 * n2 + k);
  for (size_t ij = 0; ij < (size_t)n0 * n1; ++ij) l2.push_back(ij * n2);
  fft_lines(p0, box, l0.data(), (int)l0.size(), (size_t)n1 * n2, s, sign);
  fft_lines(p1, box, l1.data(), (int)l1.size(), (size_t)n2, s, sign);
  fft_lines(p2, box, l2.data(), (int)l2.size(), 1, s, sign);
  if (sign < 0) {
    const double sc = 1.0 / ((double)n0 * n1 * n2);
    for (size_t f = 0; f < (size_t)n0 * n1 * n2; ++f) box[f] *= sc;
  }
  return 0;
}

}  // extern "C"
