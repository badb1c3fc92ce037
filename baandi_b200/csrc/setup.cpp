// Host-side operand builders: the plane-wave sphere, the alias-free FFT grid, the
// Gamma mirror maps, projector tables and the local form factor.  They restate the
// reference's setup so that a C or C++ caller without the reference engine can
// build the operator's inputs; a caller that has the engine passes its own arrays
// to bg_op_create_* instead.  CPU, FP64, called once per geometry.
//
// Reference (paths inside the reference project):
//   cell inverse / volume   crates/dft-geometry/src/lib.rs:46-94
//   sphere + sort           crates/dft-basis/src/lib.rs:55-74, 96-120, 233-265
//   grid                    crates/dft-basis/src/lib.rs:414-455
//   mirror maps             crates/dft-basis/src/half.rs:41-99
//   radial quadrature       crates/dft-upf/src/radial.rs:58-117, 246-344
//   real harmonics          crates/dft-upf/src/radial.rs:172-240
//   projector table         crates/dft-physics/src/hamiltonian.rs:2605-2760, 57-63
//   local form factor       crates/dft-upf/src/radial.rs:246-305
//
// Built with -ffp-contract=off: the |G|^2 values decide the basis ORDER (sort by
// |G|^2, ties by Miller index), so they are formed with the reference's operation
// order and no fused multiply-add.
#include "bg_internal.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <map>
#include <numeric>
#include <unordered_map>
#include <vector>

namespace bg {

static const double kTau = 6.283185307179586;
static const double kPi = 3.141592653589793;

int cell_init(const double rows[9], Cell* c) {
  for (int i = 0; i < 9; ++i)
    if (!std::isfinite(rows[i])) return BG_EINVAL;
  double a[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) a[i][j] = rows[j * 3 + i];  // columns are lattice vectors
  double scale = 0.0;
  for (auto& r : a)
    for (double x : r) scale = std::max(scale, std::fabs(x));
  if (scale == 0.0) return BG_EINVAL;
  double m[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) m[i][j] = a[i][j] / scale;
  const double c00 = m[1][1] * m[2][2] - m[1][2] * m[2][1];
  const double c01 = m[1][2] * m[2][0] - m[1][0] * m[2][2];
  const double c02 = m[1][0] * m[2][1] - m[1][1] * m[2][0];
  const double det = m[0][0] * c00 + m[0][1] * c01 + m[0][2] * c02;
  if (std::fabs(det) <= 1e-12) return BG_EINVAL;
  double inv[3][3];
  inv[0][0] = c00 / det;
  inv[1][0] = c01 / det;
  inv[2][0] = c02 / det;
  inv[0][1] = (m[0][2] * m[2][1] - m[0][1] * m[2][2]) / det;
  inv[1][1] = (m[0][0] * m[2][2] - m[0][2] * m[2][0]) / det;
  inv[2][1] = (m[0][1] * m[2][0] - m[0][0] * m[2][1]) / det;
  inv[0][2] = (m[0][1] * m[1][2] - m[0][2] * m[1][1]) / det;
  inv[1][2] = (m[0][2] * m[1][0] - m[0][0] * m[1][2]) / det;
  inv[2][2] = (m[0][0] * m[1][1] - m[0][1] * m[1][0]) / det;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      inv[i][j] /= scale;
      c->lattice[i][j] = a[i][j];
    }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) c->recip[i][j] = kTau * inv[j][i];
  c->volume = ((std::fabs(det) * scale) * scale) * scale;
  return BG_OK;
}

static void wrap_fractional(const double in[3], double out[3]) {
  for (int i = 0; i < 3; ++i) {
    const double x = in[i];
    out[i] = (x >= -0.5 && x < 0.5) ? x : x - std::floor(x + 0.5);
  }
}

int basis_build(const Cell& cell, double ecut, const double kfrac_in[3], Basis* out) {
  if (!(ecut > 0.0) || !std::isfinite(ecut)) return BG_EINVAL;
  double kf[3];
  wrap_fractional(kfrac_in, kf);
  const auto& b = cell.recip;
  double kc[3];
  for (int i = 0; i < 3; ++i) kc[i] = (b[i][0] * kf[0] + b[i][1] * kf[1]) + b[i][2] * kf[2];
  const double radius = std::sqrt(2.0 * ecut * (1.0 + 1e-12));
  int bounds[3];
  for (int i = 0; i < 3; ++i) {
    const double nrm = std::hypot(std::hypot(cell.lattice[0][i], cell.lattice[1][i]), cell.lattice[2][i]);
    bounds[i] = (int)(std::ceil(nrm * radius / kTau) + 1.0) + 1;
  }
  struct Entry {
    int m[3];
    double c[3];
    double n2;
  };
  std::vector<Entry> list;
  const double limit = ecut * (1.0 + 1e-12);
  for (int m0 = -bounds[0]; m0 <= bounds[0]; ++m0)
    for (int m1 = -bounds[1]; m1 <= bounds[1]; ++m1)
      for (int m2 = -bounds[2]; m2 <= bounds[2]; ++m2) {
        Entry e;
        e.m[0] = m0;
        e.m[1] = m1;
        e.m[2] = m2;
        for (int i = 0; i < 3; ++i) e.c[i] = (b[i][0] * (double)m0 + b[i][1] * (double)m1) + b[i][2] * (double)m2;
        e.n2 = (e.c[0] * e.c[0] + e.c[1] * e.c[1]) + e.c[2] * e.c[2];
        double q[3];
        for (int i = 0; i < 3; ++i) q[i] = e.c[i] + kc[i];
        const double q2 = (q[0] * q[0] + q[1] * q[1]) + q[2] * q[2];
        if (0.5 * q2 <= limit) list.push_back(e);
      }
  std::sort(list.begin(), list.end(), [](const Entry& x, const Entry& y) {
    if (x.n2 != y.n2) return x.n2 < y.n2;
    return std::lexicographical_compare(x.m, x.m + 3, y.m, y.m + 3);
  });
  out->npw = (int64_t)list.size();
  out->miller.resize(3 * list.size());
  out->kpg.resize(3 * list.size());
  out->kpg2.resize(list.size());
  for (size_t g = 0; g < list.size(); ++g) {
    double q[3];
    for (int i = 0; i < 3; ++i) {
      out->miller[3 * g + i] = list[g].m[i];
      q[i] = list[g].c[i] + kc[i];
      out->kpg[3 * g + i] = q[i];
    }
    out->kpg2[g] = (q[0] * q[0] + q[1] * q[1]) + q[2] * q[2];
  }
  for (int i = 0; i < 3; ++i) out->kfrac[i] = kf[i];
  return BG_OK;
}

static bool smooth(int n) {
  for (int p : {2, 3, 5})
    while (n % p == 0) n /= p;
  return n == 1;
}

int grid_dims(const Cell& cell, double ecut, int dims[3], int required[3]) {
  Basis dens;
  const double k0[3] = {0, 0, 0};
  int rc = basis_build(cell, 4.0 * ecut, k0, &dens);
  if (rc) return rc;
  for (int i = 0; i < 3; ++i) required[i] = 1;
  for (int64_t g = 0; g < dens.npw; ++g)
    for (int i = 0; i < 3; ++i) required[i] = std::max(required[i], 2 * std::abs(dens.miller[3 * g + i]) + 1);
  for (int i = 0; i < 3; ++i) {
    int d = required[i];
    while (!smooth(d)) ++d;
    dims[i] = d;
  }
  return BG_OK;
}

int fft_index(const int32_t* miller, int64_t npw, const int dims[3], bool gamma, int64_t* flat) {
  for (int64_t g = 0; g < npw; ++g) {
    int64_t idx[3];
    for (int i = 0; i < 3; ++i) {
      const int64_t n = dims[i], m = miller[3 * g + i];
      if (gamma && (m < -(n / 2) || m > (n - 1) / 2)) return BG_ESHAPE;
      idx[i] = ((m % n) + n) % n;
    }
    flat[g] = (idx[0] * dims[1] + idx[1]) * dims[2] + idx[2];
  }
  std::vector<int64_t> s(flat, flat + npw);
  std::sort(s.begin(), s.end());
  if (std::adjacent_find(s.begin(), s.end()) != s.end()) return BG_ESHAPE;
  return BG_OK;
}

int half_sphere(const int32_t* miller, int64_t npw, std::vector<int64_t>* plus, std::vector<int64_t>* minus) {
  if (npw < 1 || miller[0] != 0 || miller[1] != 0 || miller[2] != 0) return BG_ESHAPE;
  std::map<std::array<int, 3>, int64_t> lookup;
  for (int64_t g = 0; g < npw; ++g) lookup[{miller[3 * g], miller[3 * g + 1], miller[3 * g + 2]}] = g;
  if ((int64_t)lookup.size() != npw) return BG_ESHAPE;
  plus->assign(1, 0);
  minus->assign(1, 0);
  for (int64_t g = 0; g < npw; ++g) {
    const std::array<int, 3> m = {miller[3 * g], miller[3 * g + 1], miller[3 * g + 2]};
    auto it = lookup.find({-m[0], -m[1], -m[2]});
    if (it == lookup.end()) return BG_ESHAPE;
    if (m > std::array<int, 3>{0, 0, 0}) {
      plus->push_back(g);
      minus->push_back(it->second);
    }
  }
  if ((int64_t)(2 * plus->size() - 1) != npw) return BG_ESHAPE;
  return BG_OK;
}

// --------------------------------------------------------------------- radial
// Composite Simpson 1/3 in the mesh index with a final 3/8 panel for even n, panel
// sums Kahan-compensated (radial.rs:58-81).
template <class F>
static double integrate(int n, F f) {
  if (n < 2) return 0.0;
  if (n == 2) return (f(0) + f(1)) * 0.5;
  const int last = (n % 2 == 0) ? n - 4 : n - 1;
  double sum = 0.0, corr = 0.0;
  auto add = [&](double x) {
    const double y = x - corr;
    const double t = sum + y;
    corr = (t - sum) - y;
    sum = t;
  };
  for (int i = 0; i < last; i += 2) add((f(i) + 4.0 * f(i + 1) + f(i + 2)) / 3.0);
  if (n % 2 == 0) add(3.0 * (f(last) + 3.0 * f(last + 1) + 3.0 * f(last + 2) + f(last + 3)) / 8.0);
  return sum;
}

// Spherical Bessel j_l, l <= 3: power series below x = 4, upward recurrence above
// (radial.rs:89-117).
static double bessel(int l, double x) {
  if (x < 4.0) {
    double term = 1.0;
    for (int k = 1; k <= l; ++k) term *= x / (double)(2 * k + 1);
    double sum = term;
    for (int k = 1; k < 80; ++k) {
      term *= -x * x / (double)(2 * k * (2 * l + 2 * k + 1));
      sum += term;
      if (std::fabs(term) <= 2.220446049250313e-16 * std::fabs(sum)) break;
    }
    return sum;
  }
  const double s = std::sin(x), c = std::cos(x);
  double prev = s / x;
  if (l == 0) return prev;
  double cur = (prev - c) / x;
  for (int k = 1; k < l; ++k) {
    const double next = (double)(2 * k + 1) / x * cur - prev;
    prev = cur;
    cur = next;
  }
  return cur;
}

// Every real harmonic up to lmax at out[l*l+l+m] (radial.rs:172-240).
static void real_harmonics(int lmax, const double d[3], double* out) {
  const double norm = std::hypot(std::hypot(d[0], d[1]), d[2]);
  const double z = std::min(1.0, std::max(-1.0, d[2] / norm));
  const double phi = std::atan2(d[1], d[0]);
  for (int l = 0; l <= lmax; ++l)
    for (int m = -l; m <= l; ++m) {
      const int a = std::abs(m);
      double p = 1.0;
      for (int k = 1; k <= a; ++k) p *= -(double)(2 * k - 1) * std::sqrt((1.0 - z) * (1.0 + z));
      if (l > a) {
        double prev = p;
        p *= (double)(2 * a + 1) * z;
        for (int k = a + 2; k <= l; ++k) {
          const double next = ((double)(2 * k - 1) * z * p - (double)(k + a - 1) * prev) / (double)(k - a);
          prev = p;
          p = next;
        }
      }
      double ratio = 1.0;
      for (int k = l - a + 1; k <= l + a; ++k) ratio /= (double)k;
      const double nrm = std::sqrt((double)(2 * l + 1) / (4.0 * kPi) * ratio);
      double ang = 1.0;
      if (m != 0) {
        const double sign = (a % 2 == 0) ? 1.0 : -1.0;
        ang = std::sqrt(2.0) * sign * (m < 0 ? std::sin((double)a * phi) : std::cos((double)a * phi));
      }
      out[l * l + l + m] = nrm * p * ang;
    }
}

static double projector_transform(const Species& s, int i, double q) {
  const int n = s.ulen[i];
  const int l = s.l[i];
  const double* u = s.u[i];
  return 4.0 * kPi * integrate(n, [&](int k) { return s.r[k] * u[k] * bessel(l, q * s.r[k]) * s.rab[k]; });
}

int projector_count(int nspecies, const Species* sp, int* nproj, int* natoms) {
  int np = 0, na = 0;
  for (int s = 0; s < nspecies; ++s) {
    int per = 0;
    for (int i = 0; i < sp[s].nbeta; ++i) {
      if (sp[s].l[i] < 0 || sp[s].l[i] > 3) return BG_EINVAL;
      per += 2 * sp[s].l[i] + 1;
    }
    np += per * sp[s].natoms;
    na += sp[s].natoms;
  }
  *nproj = np;
  *natoms = na;
  return BG_OK;
}

int projectors_build(double volume, int64_t npw, const double* kpg, const double* kpg2, int nspecies,
                     const Species* sp, std::complex<double>* table, int32_t* channels, double* couplings) {
  if (!(volume > 0.0)) return BG_EINVAL;
  const double vr = std::sqrt(volume);
  int64_t col = 0;
  int atom = 0;
  size_t coff = 0;
  for (int si = 0; si < nspecies; ++si) {
    const Species& s = sp[si];
    const int nb = s.nbeta;
    for (int i = 0; i < nb; ++i)
      for (int j = 0; j < nb; ++j)
        if (s.l[i] != s.l[j] && s.dij[i * nb + j] != 0.0) return BG_EINVAL;
    struct Ch {
      int i, l, m;
    };
    std::vector<Ch> ch;
    int lmax = 0;
    for (int i = 0; i < nb; ++i) {
      lmax = std::max(lmax, s.l[i]);
      for (int m = -s.l[i]; m <= s.l[i]; ++m) ch.push_back({i, s.l[i], m});
    }
    const int nc = (int)ch.size();
    // factors (pref * Y) * F / sqrt(Omega), radial transforms cached per |k+G|^2
    std::vector<std::complex<double>> fac((size_t)nc * npw);
    std::unordered_map<uint64_t, size_t> cache;
    std::vector<double> radial;
    std::vector<double> ylm((lmax + 1) * (lmax + 1));
    for (int64_t g = 0; g < npw; ++g) {
      uint64_t key;
      std::memcpy(&key, &kpg2[g], sizeof key);
      size_t slot;
      auto it = cache.find(key);
      if (it == cache.end()) {
        slot = cache.size();
        cache.emplace(key, slot);
        const double q = std::sqrt(kpg2[g]);
        for (int i = 0; i < nb; ++i) radial.push_back(projector_transform(s, i, q));
      } else {
        slot = it->second;
      }
      double dir[3] = {kpg[3 * g], kpg[3 * g + 1], kpg[3 * g + 2]};
      if (kpg2[g] == 0.0) {
        dir[0] = 0.0;
        dir[1] = 0.0;
        dir[2] = 1.0;
      }
      real_harmonics(lmax, dir, ylm.data());
      for (int c = 0; c < nc; ++c) {
        std::complex<double> pref(1.0, 0.0);
        for (int k = 0; k < ch[c].l; ++k) pref *= std::complex<double>(0.0, -1.0);
        const double y = ylm[ch[c].l * ch[c].l + ch[c].l + ch[c].m];
        fac[(size_t)c * npw + g] = ((pref * y) * radial[slot * nb + ch[c].i]) / vr;
      }
    }
    std::vector<double> coupling((size_t)nc * nc, 0.0);
    for (int a = 0; a < nc; ++a)
      for (int b = 0; b < nc; ++b)
        if (ch[a].l == ch[b].l && ch[a].m == ch[b].m) coupling[(size_t)a * nc + b] = s.dij[ch[a].i * nb + ch[b].i];
    // every atom's columns on its own host thread; the phase of (atom, G) is formed once
    // for all of the atom's channels (the same arithmetic per element as one by one)
    int bad = 0;
#pragma omp parallel for schedule(dynamic) reduction(| : bad)
    for (int at = 0; at < s.natoms; ++at) {
      const double* tau = s.positions + 3 * at;
      std::vector<std::complex<double>> ph((size_t)npw);
      for (int64_t g = 0; g < npw; ++g) {
        const double ang = (kpg[3 * g] * tau[0] + kpg[3 * g + 1] * tau[1]) + kpg[3 * g + 2] * tau[2];
        ph[(size_t)g] = std::complex<double>(std::cos(-ang), std::sin(-ang));
      }
      for (int c = 0; c < nc; ++c) {
        std::complex<double>* out = table + (size_t)(col + (int64_t)at * nc + c) * npw;
        for (int64_t g = 0; g < npw; ++g) {
          const std::complex<double> v = fac[(size_t)c * npw + g] * ph[(size_t)g];
          bad |= (!std::isfinite(v.real()) || !std::isfinite(v.imag())) ? 1 : 0;
          out[g] = v;
        }
      }
    }
    if (bad) return BG_ENONFINITE;
    for (int at = 0; at < s.natoms; ++at) {
      col += nc;
      channels[atom++] = nc;
      std::copy(coupling.begin(), coupling.end(), couplings + coff);
      coff += coupling.size();
    }
  }
  return BG_OK;
}

int local_form_factor(const Species& s, double volume, int64_t n, const double* g, double* out) {
  const double end = s.r[s.mesh - 1];
  const double limit = std::min(end, 10.0);
  int npt = 0;
  while (npt < s.mesh && s.r[npt] <= limit) ++npt;
  if (npt < 2) return BG_EINVAL;
  std::vector<double> shortv(npt);
  for (int i = 0; i < npt; ++i) shortv[i] = s.r[i] * s.r[i] * s.local[i] + s.z * s.r[i] * std::erf(s.r[i]);
  for (int64_t k = 0; k < n; ++k) {
    const double q = g[k];
    const double integral = integrate(npt, [&](int i) { return shortv[i] * bessel(0, q * s.r[i]) * s.rab[i]; });
    if (q == 0.0)
      out[k] = 4.0 * kPi / volume * integral + kPi * s.z / volume;
    else
      out[k] = 4.0 * kPi / volume * (integral - s.z * std::exp(-q * q / 4.0) / (q * q));
  }
  return BG_OK;
}

// rho_atom(|G|) / Omega of PP_RHOATOM samples f (4 pi r^2 rho(r)): the integral of
// f j0(q r) over the mesh (Simpson in the index with rab, j0 = 1 at q = 0), divided by the
// volume; the exact per-shell quadrature of the atomic start density.  The q values run
// on the host threads, each integral in the mesh's fixed order.
int atomic_charge_transform(int mesh, const double* r, const double* rab, const double* f, double volume,
                            int64_t n, const double* q, double* out) {
  if (mesh < 2) return BG_EINVAL;
  for (int i = 0; i < mesh; ++i)
    if (!std::isfinite(r[i]) || !std::isfinite(rab[i]) || !std::isfinite(f[i])) return BG_ENONFINITE;
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < n; ++k) {
    const double qk = q[k];
    out[k] = integrate(mesh, [&](int i) { return f[i] * (qk == 0.0 ? 1.0 : bessel(0, qk * r[i])) * rab[i]; }) /
             volume;
  }
  return BG_OK;
}

// Ewald ion-ion energy of point charges in a neutralising background (Ha), the
// standard split with eta = sqrt(pi) / Omega^(1/3) (the reference's default scheme,
// crates/dft-physics/src/ewald.rs:1-10, 376-381): real-space erfc sum over lattice
// images, reciprocal sum (2 pi / Omega) exp(-G^2 / 4 eta^2) / G^2 |S(G)|^2, the self
// term -eta / sqrt(pi) sum Z^2 and the background -pi (sum Z)^2 / (2 eta^2 Omega).
// Both sums run to exp(-t^2) with t = 6.5 (terms below 1e-18 of the leading ones),
// widened by the cell's circumradius so that every pair is covered; long double
// accumulation.
int ewald_energy(const Cell& cell, int natoms, const double* pos, const double* charge, double* out) {
  if (natoms < 1) return BG_EINVAL;
  const double omega = cell.volume;
  const double eta = std::sqrt(kPi) / std::cbrt(omega);
  const double t = 6.5;
  double rho = 0.0, rho_g = 0.0;  // half the sum of the cell (reciprocal cell) edge lengths
  for (int j = 0; j < 3; ++j) {
    rho += 0.5 * std::sqrt(cell.lattice[0][j] * cell.lattice[0][j] + cell.lattice[1][j] * cell.lattice[1][j] +
                           cell.lattice[2][j] * cell.lattice[2][j]);
    rho_g += 0.5 * std::sqrt(cell.recip[0][j] * cell.recip[0][j] + cell.recip[1][j] * cell.recip[1][j] +
                             cell.recip[2][j] * cell.recip[2][j]);
  }
  const double r_cut = t / eta + 2.0 * rho;
  const double g_cut = 2.0 * eta * t + 2.0 * rho_g;
  // images n with |n . A| <= r_cut: |n_j| <= r_cut |b_j| / (2 pi)
  int nr[3], ng[3];
  for (int j = 0; j < 3; ++j) {
    const double bj = std::sqrt(cell.recip[0][j] * cell.recip[0][j] + cell.recip[1][j] * cell.recip[1][j] +
                                cell.recip[2][j] * cell.recip[2][j]);
    const double aj = std::sqrt(cell.lattice[0][j] * cell.lattice[0][j] + cell.lattice[1][j] * cell.lattice[1][j] +
                                cell.lattice[2][j] * cell.lattice[2][j]);
    nr[j] = (int)std::ceil(r_cut * bj / kTau) + 1;
    ng[j] = (int)std::ceil(g_cut * aj / kTau) + 1;
  }
  long double real = 0.0L, recip = 0.0L;
  double zsum = 0.0, z2sum = 0.0;
  for (int i = 0; i < natoms; ++i) {
    zsum += charge[i];
    z2sum += charge[i] * charge[i];
  }
  // the image sums of the pairs on the host threads, then added in pair order (the same
  // result as one thread)
  std::vector<long double> pair((size_t)natoms * natoms);
#pragma omp parallel for schedule(dynamic)
  for (int i = 0; i < natoms; ++i)
    for (int j = 0; j < natoms; ++j) {
      const double d0[3] = {pos[3 * j] - pos[3 * i], pos[3 * j + 1] - pos[3 * i + 1], pos[3 * j + 2] - pos[3 * i + 2]};
      long double acc = 0.0L;
      for (int a = -nr[0]; a <= nr[0]; ++a)
        for (int b = -nr[1]; b <= nr[1]; ++b)
          for (int c = -nr[2]; c <= nr[2]; ++c) {
            double d[3];
            for (int x = 0; x < 3; ++x)
              d[x] = d0[x] + a * cell.lattice[x][0] + b * cell.lattice[x][1] + c * cell.lattice[x][2];
            const double r = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            if (r > r_cut || (i == j && a == 0 && b == 0 && c == 0)) continue;
            acc += std::erfc(eta * r) / r;
          }
      pair[(size_t)i * natoms + j] = acc;
    }
  for (int i = 0; i < natoms; ++i)
    for (int j = 0; j < natoms; ++j) real += 0.5L * charge[i] * charge[j] * pair[(size_t)i * natoms + j];
  for (int a = -ng[0]; a <= ng[0]; ++a)
    for (int b = -ng[1]; b <= ng[1]; ++b)
      for (int c = -ng[2]; c <= ng[2]; ++c) {
        if (a == 0 && b == 0 && c == 0) continue;
        double g[3];
        for (int x = 0; x < 3; ++x) g[x] = a * cell.recip[x][0] + b * cell.recip[x][1] + c * cell.recip[x][2];
        const double g2 = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
        if (g2 > g_cut * g_cut) continue;
        double sr = 0.0, si = 0.0;
        for (int i = 0; i < natoms; ++i) {
          const double ph = g[0] * pos[3 * i] + g[1] * pos[3 * i + 1] + g[2] * pos[3 * i + 2];
          sr += charge[i] * std::cos(ph);
          si += charge[i] * std::sin(ph);
        }
        recip += (long double)(std::exp(-g2 / (4.0 * eta * eta)) / g2 * (sr * sr + si * si));
      }
  const long double e = real + (long double)(2.0 * kPi / omega) * recip - (long double)(eta / std::sqrt(kPi) * z2sum) -
                        (long double)(kPi * zsum * zsum / (2.0 * eta * eta * omega));
  *out = (double)e;
  return std::isfinite(*out) ? BG_OK : BG_ENONFINITE;
}

}  // namespace bg
